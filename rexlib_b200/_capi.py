"""ctypes binding of librexlib_b200.so (the C-ABI declared in include/rexlib_b200.h).

The library is built in-tree (``rexlib_b200/_lib``) by ``rexlib_b200.build``.
Loading fails loudly when it is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# REXLIB_B200_LIBRARY names another build of the same library (for example a
# debug build); the in-tree build is the default.
LIBRARY = os.environ.get("REXLIB_B200_LIBRARY") or os.path.join(HERE, "_lib", "librexlib_b200.so")

OK = 0
INVALID_ARGUMENT = 1
UNSUPPORTED = 2
CUDA_ERROR = 3
WORKSPACE_TOO_SMALL = 4

WINDOW_BOX = 0
WINDOW_TRIANGLE = 1
WINDOW_KAISER_BESSEL = 2

INSERT_THROUGHPUT = 0
INSERT_DETERMINISTIC = 1


class GriddingWindowC(ctypes.Structure):
    _fields_ = [("profile", ctypes.c_int32), ("half_width", ctypes.c_double), ("shape", ctypes.c_double)]


class CtfOpticsC(ctypes.Structure):
    _fields_ = [
        ("voltage", ctypes.c_double),
        ("spherical_aberration", ctypes.c_double),
        ("amplitude_contrast", ctypes.c_double),
    ]


class BatchStrides(ctypes.Structure):
    _fields_ = [("volume", ctypes.c_int64), ("particle", ctypes.c_int64)]


class Insertion(ctypes.Structure):
    _fields_ = [
        ("numerator_out", ctypes.c_void_p),
        ("denominator_out", ctypes.c_void_p),
        ("numerator_in", ctypes.c_void_p),
        ("denominator_in", ctypes.c_void_p),
        ("slices", ctypes.c_void_p),
        ("transforms", ctypes.c_void_p),
        ("radial_weights", ctypes.c_void_p),
        ("slice_strides", BatchStrides),
        ("transform_strides", BatchStrides),
        ("radial_strides", BatchStrides),
        ("volume_count", ctypes.c_int64),
        ("slices_per_volume", ctypes.c_int64),
        ("slice_extent", ctypes.c_int64),
        ("volume_extent", ctypes.c_int64),
        ("window", GriddingWindowC),
        ("mode", ctypes.c_int32),
        ("workspace", ctypes.c_void_p),
        ("workspace_bytes", ctypes.c_size_t),
        ("element_type", ctypes.c_int32),
    ]


class Standardization(ctypes.Structure):
    _fields_ = [
        ("result", ctypes.c_void_p),
        ("value", ctypes.c_void_p),
        ("keys", ctypes.c_void_p),
        ("images_per_key", ctypes.c_int64),
        ("batch", ctypes.c_int64),
        ("rank", ctypes.c_int32),
        ("extents", ctypes.c_int64 * 3),
        ("radius", ctypes.c_double),
        ("lower_bound", ctypes.c_double),
        ("upper_bound", ctypes.c_double),
        ("statistics", ctypes.c_void_p),
    ]


class CtfEpilogue(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32),
        ("ctf", ctypes.c_void_p),
        ("ctf_stride", ctypes.c_int64),
        ("voltage", ctypes.c_void_p),
        ("optics", CtfOpticsC),
        ("pixel_size", ctypes.c_double),
        ("weights", ctypes.c_void_p),
    ]


class InsertionJob(ctypes.Structure):
    _fields_ = [("insertion", Insertion), ("extra", ctypes.c_void_p), ("extra_strides", BatchStrides)]


class TileConfig(ctypes.Structure):
    _fields_ = [("cells", ctypes.c_int32), ("min_hits", ctypes.c_int32), ("max_hits", ctypes.c_int32)]


class Conv3dArgs(ctypes.Structure):
    _fields_ = [
        ("sources", ctypes.c_int32),
        ("inputs", ctypes.c_void_p * 2),
        ("input_channels", ctypes.c_int32 * 2),
        ("input_strides", ctypes.c_int32 * 2),
        ("depth", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("weights", ctypes.c_void_p),
        ("bias", ctypes.c_void_p),
        ("output_channels", ctypes.c_int32),
        ("epilogue", ctypes.c_int32),
        ("outputs", ctypes.c_void_p * 2),
        ("output_strides", ctypes.c_int32 * 2),
        ("output_split", ctypes.c_int32),
        ("masks", ctypes.c_void_p * 2),
        ("mask_strides", ctypes.c_int32 * 2),
        ("error", ctypes.c_void_p),
        ("wait_limit_ns", ctypes.c_int64),
    ]


class Conv3dWgradArgs(ctypes.Structure):
    _fields_ = [
        ("sources", ctypes.c_int32),
        ("inputs", ctypes.c_void_p * 2),
        ("input_channels", ctypes.c_int32 * 2),
        ("input_strides", ctypes.c_int32 * 2),
        ("depth", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("output_grad", ctypes.c_void_p),
        ("output_channels", ctypes.c_int32),
        ("output_grad_stride", ctypes.c_int32),
        ("weight_grad", ctypes.c_void_p),
        ("bias_grad", ctypes.c_void_p),
        ("error", ctypes.c_void_p),
        ("wait_limit_ns", ctypes.c_int64),
    ]


KIND_PLAIN = 0
KIND_CTF = 1
KIND_WEIGHTED = 2

FLOAT32 = 0
FLOAT64 = 1
COMPLEX64 = 2
COMPLEX128 = 3

WIENER_REGULARIZED = 0
WIENER_THRESHOLD = 1


class RexlibB200Error(RuntimeError):
    """An error status returned by the C-ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_lib: ctypes.CDLL | None = None

# Exported names and their (argtypes, restype).
SIGNATURES: dict[str, tuple[list, object]] = {
    "rexlib_b200_last_error": ([], ctypes.c_char_p),
    "rexlib_b200_abi_version": ([], ctypes.c_int32),
    "rexlib_b200_insertion_workspace_size": ([ctypes.POINTER(Insertion), ctypes.POINTER(ctypes.c_size_t)],
                                             ctypes.c_int32),
    "rexlib_b200_insertion_launches": ([ctypes.POINTER(Insertion), ctypes.POINTER(ctypes.c_int32)], ctypes.c_int32),
    "rexlib_b200_l2_reduction_run": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_uint32, ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_shared_atomic_run": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32,
                                       ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_insert_slices": ([ctypes.POINTER(Insertion), ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_insert_weighted_slices": ([ctypes.POINTER(Insertion), ctypes.c_void_p, BatchStrides,
                                            ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_insert_ctf_slices": ([ctypes.POINTER(Insertion), ctypes.c_void_p, BatchStrides, CtfOpticsC,
                                       ctypes.c_double, ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_insert_ctf_slices_fixed_scratch": ([ctypes.POINTER(Insertion), ctypes.c_void_p, BatchStrides,
                                                     CtfOpticsC, ctypes.c_double, ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_batched_insertion_workspace_size": ([ctypes.POINTER(InsertionJob), ctypes.c_int32, ctypes.c_int32,
                                                      ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int32),
    "rexlib_b200_batched_insert": ([ctypes.POINTER(InsertionJob), ctypes.c_int32, ctypes.c_int32, CtfOpticsC,
                                    ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
                                   ctypes.c_int32),
    "rexlib_b200_batched_tuning": ([ctypes.POINTER(InsertionJob), ctypes.c_int32, ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(TileConfig)], ctypes.c_int32),
    "rexlib_b200_batched_insertion_launches": ([ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int32),
    "rexlib_b200_conv3d": ([ctypes.POINTER(Conv3dArgs), ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_conv3d_wgrad": ([ctypes.POINTER(Conv3dWgradArgs), ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_rfft3": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_fsc": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p],
                        ctypes.c_int32),
    "rexlib_b200_prior_wiener": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                  ctypes.c_double, ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_blob_spectrum": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double,
                                   ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_phantom_slices": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                                    ctypes.c_void_p, ctypes.c_void_p, CtfOpticsC, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_uint64, ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_unet_create": ([ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int32),
    "rexlib_b200_unet_destroy": ([ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_unet_parameter_count": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int32),
    "rexlib_b200_unet_copy": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                              ctypes.c_int32),
    "rexlib_b200_unet_layer": ([ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64),
                                ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)], ctypes.c_int32),
    "rexlib_b200_unet_tensor": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p],
                                ctypes.c_int32),
    "rexlib_b200_unet_forward": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                                 ctypes.c_int32),
    "rexlib_b200_unet_backward": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                                  ctypes.c_int32),
    "rexlib_b200_unet_adam_step": ([ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_unet_error": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int32),
    "rexlib_b200_standardize_background": ([ctypes.POINTER(Standardization), ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_rfft2": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                           ctypes.POINTER(CtfEpilogue), ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_standardize_rfft2": ([ctypes.c_void_p, ctypes.POINTER(Standardization), ctypes.POINTER(CtfEpilogue),
                                       ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_irfft2": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p],
                           ctypes.c_int32),
    "rexlib_b200_irfft3_workspace_size": ([ctypes.c_int64, ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int32),
    "rexlib_b200_irfft3": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_size_t,
                            ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_wiener_irfft3": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                   ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
                                  ctypes.c_int32),
    "rexlib_b200_fill": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p],
                         ctypes.c_int32),
    "rexlib_b200_add": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                         ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p], ctypes.c_int32),
    "rexlib_b200_divide": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                            ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p], ctypes.c_int32),
}


def load() -> ctypes.CDLL:
    """Load the library, binding every exported entry point."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            raise ImportError(
                f"{LIBRARY} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "or `make -C rexlib_b200/csrc`; rexlib_b200 has no CPU fallback")
        lib = ctypes.CDLL(LIBRARY)
        for name, (argtypes, restype) in SIGNATURES.items():
            f = getattr(lib, name)
            f.argtypes = argtypes
            f.restype = restype
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != OK:
        message = load().rexlib_b200_last_error().decode()
        raise RexlibB200Error(status, message)
