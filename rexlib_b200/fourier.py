"""rexlib's real FFTs and the Wiener step on the B200 backend.

Mirrors the functional FFTs of the reference (include/rexlib/functional/
fourier.hpp: rfft2, irfft2, irfft3 with the default backward normalisation)
over the C-ABI of librexlib_b200.so, for square images and cubic volumes of
the supported extents. `rfft2_ctf` is the R2C with the CTF epilogue,
`standardize_rfft2_ctf` the background standardization fused in front of it,
and `wiener_irfft3` the divide of an insertion's accumulators fused into the
C2R; none has a counterpart operation in the reference.
"""

from __future__ import annotations

import ctypes
import math

import torch

from . import _capi
from .em import CtfOptics, _check_device, _resolve_bounds, _stream

__all__ = ["irfft2", "irfft3", "rfft2", "rfft2_ctf", "standardize_rfft2_ctf", "wiener_irfft3"]

EXTENTS = (32, 64, 96, 128, 160, 192, 200, 256)


def _square_images(x: torch.Tensor, name: str) -> tuple[int, int]:
    if x.ndim < 2 or x.shape[-1] != x.shape[-2]:
        raise ValueError(f"{name} must hold square images in its last two axes")
    n = x.shape[-1]
    return math.prod(x.shape[:-2]), n


def rfft2(images: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """Unnormalised R2C of float32 images (..., n, n) into (..., n, n//2+1)."""
    _check_device("images", images, torch.float32)
    batch, n = _square_images(images, "images")
    x = images.contiguous()
    result = out if out is not None else torch.empty(*images.shape[:-1], n // 2 + 1, dtype=torch.complex64,
                                                     device=images.device)
    _check_device("out", result, torch.complex64)
    _capi.check(_capi.load().rexlib_b200_rfft2(ctypes.c_void_p(result.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                               batch, n, None, _stream()))
    return result


def _ctf_epilogue(images: torch.Tensor, batch: int, n: int, ctf: torch.Tensor, optics: CtfOptics,
                  pixel_size: float, voltage: torch.Tensor | None, phase_flip: bool, weights: bool):
    """The CTF epilogue descriptor of an R2C of `images` (batch images of n),
    the weights it writes (or None), and the tensors it points into."""
    _check_device("ctf", ctf, torch.float32)
    if ctf.shape[-1] != 4:
        raise ValueError("ctf must have the core axis (4)")
    c = ctf.contiguous()
    if c.numel() == 4:
        stride = 0
    elif c.numel() == 4 * batch:
        stride = 4
    else:
        raise ValueError("ctf must hold one parameter set, or one per image")
    h = n // 2 + 1
    w = torch.empty(*images.shape[:-1], h, dtype=torch.float32, device=images.device) if weights else None
    epi = _capi.CtfEpilogue()
    epi.mode = 2 if phase_flip else 1
    epi.ctf = c.data_ptr()
    epi.ctf_stride = stride
    if voltage is not None:
        _check_device("voltage", voltage, torch.float32)
        if voltage.numel() != batch:
            raise ValueError("voltage must hold one value per image")
        voltage = voltage.contiguous()
        epi.voltage = voltage.data_ptr()
    epi.optics = optics._c()
    epi.pixel_size = float(pixel_size)
    epi.weights = w.data_ptr() if w is not None else None
    return epi, w, (c, voltage)


def rfft2_ctf(images: torch.Tensor, ctf: torch.Tensor, optics: CtfOptics, pixel_size: float,
              voltage: torch.Tensor | None = None, phase_flip: bool = False, weights: bool = True):
    """R2C with the CTF epilogue: returns (c(k) X(k), c(k)^2), or with
    `phase_flip` (sign(c(k)) X(k), |c(k)|). ctf: (..., 4) per image (defocus
    U, V in angstroms, astigmatism angle, phase shift), or (4) for all."""
    _check_device("images", images, torch.float32)
    batch, n = _square_images(images, "images")
    epi, w, _keep = _ctf_epilogue(images, batch, n, ctf, optics, pixel_size, voltage, phase_flip, weights)
    x = images.contiguous()
    spectra = torch.empty(*images.shape[:-1], n // 2 + 1, dtype=torch.complex64, device=images.device)
    _capi.check(_capi.load().rexlib_b200_rfft2(ctypes.c_void_p(spectra.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                               batch, n, ctypes.byref(epi), _stream()))
    return spectra, w


def standardize_rfft2_ctf(images: torch.Tensor, key: torch.Tensor, radius: float,
                          bounds: float | tuple[float, float], ctf: torch.Tensor | None = None,
                          optics: CtfOptics | None = None, pixel_size: float = 1.0,
                          voltage: torch.Tensor | None = None, phase_flip: bool = False, weights: bool = True,
                          *, standardized: torch.Tensor | None = None, statistics: torch.Tensor | None = None,
                          out: torch.Tensor | None = None):
    """em.standardize_background_2d followed by rfft2 (with the CTF epilogue
    when `ctf` is given), in one pass over square images of 64, 128 or 256:
    the standardized images never travel through HBM unless `standardized`
    asks for them.
    The images that share a key are consecutive in the batch order: `key`
    holds one key, or one per run of batch / key.numel() images. Returns
    (spectra, weights), the weights None without a CTF or with `weights`
    false; both are bit-identical to the two separate calls'. `out`, when
    given, receives the spectra (contiguous complex64 of the spectra's
    shape)."""
    _check_device("images", images, torch.float32)
    batch, n = _square_images(images, "images")
    if not isinstance(key, torch.Tensor) or key.dtype not in (torch.uint64, torch.int64):
        raise TypeError("key must be a uint64 tensor")
    if not key.is_cuda:
        raise ValueError("key must live on a CUDA device")
    if key.numel() == 0 or batch % key.numel():
        raise ValueError("the key must hold one key, or one per equal run of consecutive images")
    lower, upper = _resolve_bounds(bounds)
    x = images.contiguous()
    keys = key.contiguous().reshape(-1)
    desc = _capi.Standardization()
    desc.value = x.data_ptr()
    desc.keys = keys.data_ptr()
    desc.images_per_key = max(1, batch // keys.numel())
    desc.batch = batch
    desc.rank = 2
    desc.extents[0] = n
    desc.extents[1] = n
    desc.radius = float(radius)
    desc.lower_bound = lower
    desc.upper_bound = upper
    if standardized is not None:
        _check_device("standardized", standardized, torch.float32)
        if standardized.shape != images.shape or not standardized.is_contiguous():
            raise ValueError("standardized must be a contiguous array of the images' shape")
        desc.result = standardized.data_ptr()
    if statistics is not None:
        if statistics.dtype != torch.float64 or not statistics.is_cuda or statistics.numel() != 2 * batch:
            raise ValueError("statistics must be a float64 CUDA tensor of batch x 2 elements")
        desc.statistics = statistics.data_ptr()
    epi, w, _keep = None, None, None
    if ctf is not None:
        if optics is None:
            raise ValueError("the CTF epilogue needs the optics")
        epi, w, _keep = _ctf_epilogue(images, batch, n, ctf, optics, pixel_size, voltage, phase_flip, weights)
    shape = (*images.shape[:-1], n // 2 + 1)
    if out is not None:
        _check_device("out", out, torch.complex64)
        if tuple(out.shape) != shape or not out.is_contiguous():
            raise ValueError(f"out must be a contiguous complex64 array of shape {shape}")
        spectra = out
    else:
        spectra = torch.empty(shape, dtype=torch.complex64, device=images.device)
    _capi.check(_capi.load().rexlib_b200_standardize_rfft2(ctypes.c_void_p(spectra.data_ptr()), ctypes.byref(desc),
                                                           ctypes.byref(epi) if epi is not None else None,
                                                           _stream()))
    return spectra, w


def irfft2(spectra: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """C2R of complex64 half spectra (..., n, n//2+1) into (..., n, n), 1/n^2."""
    _check_device("spectra", spectra, torch.complex64)
    n = spectra.shape[-2]
    if spectra.shape[-1] != n // 2 + 1:
        raise ValueError("spectra must have the core axes (n, n // 2 + 1)")
    batch = math.prod(spectra.shape[:-2])
    x = spectra.contiguous()
    result = out if out is not None else torch.empty(*spectra.shape[:-1], n, dtype=torch.float32,
                                                     device=spectra.device)
    _capi.check(_capi.load().rexlib_b200_irfft2(ctypes.c_void_p(result.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                                batch, n, _stream()))
    return result


def _workspace(extent: int, device) -> torch.Tensor:
    size = ctypes.c_size_t(0)
    _capi.check(_capi.load().rexlib_b200_irfft3_workspace_size(extent, ctypes.byref(size)))
    return torch.empty(size.value, dtype=torch.uint8, device=device)


def _volume_extent(t: torch.Tensor, name: str) -> int:
    if t.ndim != 3 or t.shape[0] != t.shape[1] or t.shape[2] != t.shape[0] // 2 + 1:
        raise ValueError(f"{name} must have the shape (N, N, N // 2 + 1)")
    return t.shape[0]


def irfft3(spectrum: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """C2R of a complex64 half spectrum (N, N, N//2+1) into (N, N, N), 1/N^3."""
    _check_device("spectrum", spectrum, torch.complex64)
    big = _volume_extent(spectrum, "spectrum")
    x = spectrum.contiguous()
    result = out if out is not None else torch.empty(big, big, big, dtype=torch.float32, device=spectrum.device)
    ws = _workspace(big, spectrum.device)
    _capi.check(_capi.load().rexlib_b200_irfft3(ctypes.c_void_p(result.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                                big, ctypes.c_void_p(ws.data_ptr()), ws.numel(), _stream()))
    return result


def wiener_irfft3(numerator: torch.Tensor, denominator: torch.Tensor, constant: float = 1e-3,
                  threshold: bool = False, out: torch.Tensor | None = None) -> torch.Tensor:
    """irfft3 of numerator / (denominator + constant), or of numerator /
    denominator where denominator > constant (0 elsewhere) with `threshold`."""
    _check_device("numerator", numerator, torch.complex64)
    _check_device("denominator", denominator, torch.float32)
    big = _volume_extent(numerator, "numerator")
    if denominator.shape != numerator.shape:
        raise ValueError("denominator must have the shape of the numerator")
    num = numerator.contiguous()
    den = denominator.contiguous()
    result = out if out is not None else torch.empty(big, big, big, dtype=torch.float32, device=numerator.device)
    ws = _workspace(big, numerator.device)
    mode = _capi.WIENER_THRESHOLD if threshold else _capi.WIENER_REGULARIZED
    _capi.check(_capi.load().rexlib_b200_wiener_irfft3(
        ctypes.c_void_p(result.data_ptr()), ctypes.c_void_p(num.data_ptr()), ctypes.c_void_p(den.data_ptr()), big, mode,
        float(constant), ctypes.c_void_p(ws.data_ptr()), ws.numel(), _stream()))
    return result
