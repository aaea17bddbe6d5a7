"""rexlib's em functional API on the B200 backend.

Mirrors ``rexlib.em`` (python/rexlib/em/_functional.py of the reference):
the same function names, parameter order and meaning, with torch CUDA
tensors standing for rexlib device arrays and the current torch stream for
the execution context's queue. Every call goes through the C-ABI of
librexlib_b200.so; nothing here computes on the host.
"""

from __future__ import annotations

import ctypes
import math
import os
from collections.abc import Sequence
from dataclasses import dataclass

import torch

from . import _capi

__all__ = [
    "standardize_background",
    "standardize_background_2d",
    "standardize_background_3d",
    "CtfOptics",
    "GriddingWindow",
    "insert_ctf_slices",
    "insert_slices",
    "insert_weighted_slices",
    "BatchedInsertion",
]


# --------------------------------------------------------------------------
# Parameters


@dataclass(frozen=True)
class GriddingWindow:
    """em::gridding_window (src/em/ops/parameters/gridding_window.cpp)."""

    profile: int
    half_width: float
    shape: float = 0.0

    @staticmethod
    def nearest() -> GriddingWindow:
        return GriddingWindow(_capi.WINDOW_BOX, 0.5, 0.0)

    @staticmethod
    def linear() -> GriddingWindow:
        return GriddingWindow(_capi.WINDOW_TRIANGLE, 1.0, 0.0)

    @staticmethod
    def kaiser_bessel(half_width: float, shape: float) -> GriddingWindow:
        if not (math.isfinite(half_width) and half_width > 0.0):
            raise ValueError(
                "gridding_window: the half-width of a Kaiser-Bessel window must be finite and positive, "
                f"but it is {half_width}.")
        if not (math.isfinite(shape) and shape >= 0.0):
            raise ValueError(
                f"gridding_window: the shape of a Kaiser-Bessel window must be finite and 0 or more, but it is {shape}.")
        return GriddingWindow(_capi.WINDOW_KAISER_BESSEL, float(half_width), float(shape))

    def _c(self) -> _capi.GriddingWindowC:
        return _capi.GriddingWindowC(self.profile, self.half_width, self.shape)


@dataclass(frozen=True)
class CtfOptics:
    """em::ctf_optics: voltage (kV), spherical aberration (mm), amplitude contrast."""

    voltage: float
    spherical_aberration: float
    amplitude_contrast: float

    def __post_init__(self):
        if not (math.isfinite(self.voltage) and self.voltage > 0.0):
            raise ValueError(f"ctf_optics: the voltage must be finite and positive, but it is {self.voltage}.")
        if not math.isfinite(self.spherical_aberration):
            raise ValueError("ctf_optics: the spherical aberration must be finite, but it is "
                             f"{self.spherical_aberration}.")
        if not (0.0 <= self.amplitude_contrast < 1.0):
            raise ValueError("ctf_optics: the amplitude contrast must lie in [0, 1), but it is "
                             f"{self.amplitude_contrast}.")

    @property
    def wavelength(self) -> float:
        """Relativistic electron wavelength in angstroms (ctf_optics.cpp:81-85)."""
        volts = self.voltage * 1e3
        return 12.2643247 / math.sqrt(volts * (1.0 + 0.978466e-6 * volts))

    def _c(self) -> _capi.CtfOpticsC:
        return _capi.CtfOpticsC(self.voltage, self.spherical_aberration, self.amplitude_contrast)


# --------------------------------------------------------------------------
# Batch planning


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check_device(name: str, t: torch.Tensor, dtype: torch.dtype) -> None:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must live on a CUDA device (rexlib_b200 runs no host fallback)")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, not {t.dtype}")


def _split(t: torch.Tensor, core: int) -> tuple[tuple[int, ...], tuple[int, ...]]:
    return tuple(t.shape[: t.ndim - core]), tuple(t.shape[t.ndim - core:])


class _BatchPlan:
    """Kept axes (the accumulators own them) and reduced axes (summed), as in
    slice_insertion_layout_plan (src/backends/cpu/plans/slice_insertion_layout_plan.cpp:81-185)."""

    def __init__(self, accumulator_batch: tuple[int, ...], input_batches: Sequence[tuple[int, ...]]):
        try:
            shape = torch.broadcast_shapes(accumulator_batch, *input_batches)
        except RuntimeError as e:
            raise ValueError(f"the batch axes of the operands do not broadcast: {e}") from None
        self.shape = tuple(shape)
        rank = len(self.shape)
        acc = (1,) * (rank - len(accumulator_batch)) + tuple(accumulator_batch)
        self.kept = [i for i in range(rank) if acc[i] != 1]
        self.reduced = [i for i in range(rank) if acc[i] == 1]
        self.volumes = math.prod(self.shape[i] for i in self.kept)
        self.particles = math.prod(self.shape[i] for i in self.reduced)

    def strides(self, t: torch.Tensor, core: int) -> tuple[torch.Tensor, _capi.BatchStrides]:
        """A view of `t` with a contiguous core, and its (volume, particle)
        strides in cores over the planned batch."""
        batch, core_shape = _split(t, core)
        if t.numel() and not t[(0,) * len(batch)].is_contiguous():
            t = t.contiguous()
        rank = len(self.shape)
        view = t.reshape((1,) * (rank - len(batch)) + tuple(t.shape)) if len(batch) < rank else t
        view = view.expand(*self.shape, *core_shape)
        view = view.permute(*self.kept, *self.reduced, *range(rank, rank + core))
        flat = view.reshape(self.volumes, self.particles, *core_shape)
        core_size = max(1, math.prod(core_shape))
        if flat.numel() and not flat[0, 0].is_contiguous():
            flat = flat.contiguous()
        sv = flat.stride(0) // core_size if self.volumes > 1 else 0
        sp = flat.stride(1) // core_size if self.particles > 1 else 0
        if (self.volumes > 1 and flat.stride(0) % core_size) or (self.particles > 1 and flat.stride(1) % core_size):
            flat = flat.contiguous()
            sv, sp = (self.particles if self.volumes > 1 else 0), (1 if self.particles > 1 else 0)
        return flat, _capi.BatchStrides(sv, sp)


def _mode(deterministic: bool | None) -> int:
    if deterministic is None:
        deterministic = os.environ.get("REXLIB_B200_DETERMINISTIC", "0") not in ("", "0", "false", "False")
    return _capi.INSERT_DETERMINISTIC if deterministic else _capi.INSERT_THROUGHPUT


# The insertions' element types (slice_insertion_rules.hpp:86-90): every
# operand float32 (complex64), or every operand float64 (complex128).
_INSERTION_TYPES = {torch.complex64: (torch.float32, _capi.FLOAT32), torch.complex128: (torch.float64, _capi.FLOAT64)}


def _insertion_real_type(numerator: torch.Tensor) -> torch.dtype:
    if not isinstance(numerator, torch.Tensor):
        raise TypeError("numerator must be a tensor")
    if numerator.dtype not in _INSERTION_TYPES:
        raise TypeError(f"numerator must be complex64 or complex128, not {numerator.dtype}")
    return _INSERTION_TYPES[numerator.dtype][0]


def _prepare_insertion(numerator, denominator, slices, transforms, radial_weights, window, numerator_out,
                       denominator_out, deterministic, extra_batches=()):
    real = _insertion_real_type(numerator)
    cplx = numerator.dtype
    _check_device("numerator", numerator, cplx)
    _check_device("denominator", denominator, real)
    _check_device("slices", slices, cplx)
    _check_device("transforms", transforms, real)
    _check_device("radial_weights", radial_weights, real)
    if numerator.ndim < 3 or numerator.shape[-1] != numerator.shape[-3] // 2 + 1 or \
            numerator.shape[-2] != numerator.shape[-3]:
        raise ValueError(f"numerator must have the core axes (N, N, N // 2 + 1), not {tuple(numerator.shape)}")
    if denominator.shape != numerator.shape:
        raise ValueError("denominator must have the shape of the numerator")
    big = numerator.shape[-3]
    if slices.ndim < 2 or slices.shape[-1] != slices.shape[-2] // 2 + 1:
        raise ValueError(f"slices must have the core axes (n, n // 2 + 1), not {tuple(slices.shape)}")
    n = slices.shape[-2]
    if transforms.ndim < 2 or tuple(transforms.shape[-2:]) != (3, 4):
        raise ValueError("transforms must have the core axes (3, 4)")
    if radial_weights.ndim < 1 or radial_weights.shape[-1] != n // 2 + 1:
        raise ValueError("radial_weights must have the core axis (n // 2 + 1)")
    if not isinstance(window, GriddingWindow):
        raise TypeError("window must be a GriddingWindow")
    acc_batch, _ = _split(numerator, 3)
    plan = _BatchPlan(acc_batch, [_split(slices, 2)[0], _split(transforms, 2)[0], _split(radial_weights, 1)[0],
                                  *extra_batches])
    if math.prod(plan.shape[i] for i in plan.kept) != math.prod(acc_batch):
        raise ValueError("the accumulators must hold every batch axis they keep")
    num_in = numerator.contiguous()
    den_in = denominator.contiguous()
    num_out = numerator_out if numerator_out is not None else torch.empty_like(num_in)
    den_out = denominator_out if denominator_out is not None else torch.empty_like(den_in)
    _check_device("numerator_out", num_out, cplx)
    _check_device("denominator_out", den_out, real)
    if num_out.shape != numerator.shape or den_out.shape != denominator.shape:
        raise ValueError("the outputs must have the shape of the accumulators")
    if not (num_out.is_contiguous() and den_out.is_contiguous()):
        raise ValueError("the outputs must be contiguous")
    sl, sl_strides = plan.strides(slices, 2)
    tr, tr_strides = plan.strides(transforms, 2)
    ra, ra_strides = plan.strides(radial_weights, 1)
    desc = _capi.Insertion()
    desc.numerator_out = num_out.data_ptr()
    desc.denominator_out = den_out.data_ptr()
    desc.numerator_in = num_in.data_ptr()
    desc.denominator_in = den_in.data_ptr()
    desc.slices = sl.data_ptr()
    desc.transforms = tr.data_ptr()
    desc.radial_weights = ra.data_ptr()
    desc.slice_strides = sl_strides
    desc.transform_strides = tr_strides
    desc.radial_strides = ra_strides
    desc.volume_count = plan.volumes
    desc.slices_per_volume = plan.particles
    desc.slice_extent = n
    desc.volume_extent = big
    desc.window = window._c()
    desc.mode = _mode(deterministic)
    desc.element_type = _INSERTION_TYPES[cplx][1]
    keep = [num_in, den_in, sl, tr, ra]
    return desc, plan, num_out, den_out, keep


def _attach_workspace(desc: _capi.Insertion, keep: list) -> None:
    lib = _capi.load()
    size = ctypes.c_size_t(0)
    _capi.check(lib.rexlib_b200_insertion_workspace_size(ctypes.byref(desc), ctypes.byref(size)))
    if size.value:
        device = torch.device("cuda", torch.cuda.current_device())
        ws = torch.empty(size.value, dtype=torch.uint8, device=device)
        keep.append(ws)
        desc.workspace = ws.data_ptr()
        desc.workspace_bytes = size.value


# --------------------------------------------------------------------------
# Insertions


def insert_slices(numerator: torch.Tensor, denominator: torch.Tensor, slices: torch.Tensor,
                  transforms: torch.Tensor, radial_weights: torch.Tensor, window: GriddingWindow,
                  context=None, numerator_out: torch.Tensor | None = None,
                  denominator_out: torch.Tensor | None = None, *, deterministic: bool | None = None
                  ) -> tuple[torch.Tensor, torch.Tensor]:
    """em.insert_slices (python/rexlib/em/_functional.py:151-205): add the
    slices into the numerator and their radial weights into the denominator.
    Pass the accumulators as the outputs to update them in place."""
    desc, plan, num_out, den_out, keep = _prepare_insertion(
        numerator, denominator, slices, transforms, radial_weights, window, numerator_out, denominator_out,
        deterministic)
    _attach_workspace(desc, keep)
    _capi.check(_capi.load().rexlib_b200_insert_slices(ctypes.byref(desc), _stream()))
    return num_out, den_out


def insert_weighted_slices(numerator: torch.Tensor, denominator: torch.Tensor, slices: torch.Tensor,
                           weights: torch.Tensor, transforms: torch.Tensor, radial_weights: torch.Tensor,
                           window: GriddingWindow, context=None, numerator_out: torch.Tensor | None = None,
                           denominator_out: torch.Tensor | None = None, *, deterministic: bool | None = None
                           ) -> tuple[torch.Tensor, torch.Tensor]:
    """em.insert_weighted_slices (python/rexlib/em/_functional.py:207-254):
    the denominator receives the weight W(k) of each frequency."""
    _check_device("weights", weights, _insertion_real_type(numerator))
    if weights.ndim < 2 or tuple(weights.shape[-2:]) != tuple(slices.shape[-2:]):
        raise ValueError("weights must have the core axes of the slices")
    desc, plan, num_out, den_out, keep = _prepare_insertion(
        numerator, denominator, slices, transforms, radial_weights, window, numerator_out, denominator_out,
        deterministic, extra_batches=[_split(weights, 2)[0]])
    w, w_strides = plan.strides(weights, 2)
    keep.append(w)
    _attach_workspace(desc, keep)
    _capi.check(_capi.load().rexlib_b200_insert_weighted_slices(ctypes.byref(desc), ctypes.c_void_p(w.data_ptr()),
                                                               w_strides, _stream()))
    return num_out, den_out


def insert_ctf_slices(numerator: torch.Tensor, denominator: torch.Tensor, slices: torch.Tensor,
                      transforms: torch.Tensor, ctf: torch.Tensor, radial_weights: torch.Tensor,
                      window: GriddingWindow, optics: CtfOptics, pixel_size: float, context=None,
                      numerator_out: torch.Tensor | None = None, denominator_out: torch.Tensor | None = None,
                      *, deterministic: bool | None = None) -> tuple[torch.Tensor, torch.Tensor]:
    """em.insert_ctf_slices (python/rexlib/em/_functional.py:256-310): the
    numerator receives c(k) times each slice and the denominator c(k)^2."""
    _check_device("ctf", ctf, _insertion_real_type(numerator))
    if ctf.ndim < 1 or ctf.shape[-1] != 4:
        raise ValueError("ctf must have the core axis (4)")
    if not isinstance(optics, CtfOptics):
        raise TypeError("optics must be a CtfOptics")
    if not (math.isfinite(pixel_size) and pixel_size > 0.0):
        raise ValueError(f"the pixel size must be finite and positive, but it is {pixel_size}.")
    desc, plan, num_out, den_out, keep = _prepare_insertion(
        numerator, denominator, slices, transforms, radial_weights, window, numerator_out, denominator_out,
        deterministic, extra_batches=[_split(ctf, 1)[0]])
    c, c_strides = plan.strides(ctf, 1)
    keep.append(c)
    _attach_workspace(desc, keep)
    _capi.check(_capi.load().rexlib_b200_insert_ctf_slices(ctypes.byref(desc), ctypes.c_void_p(c.data_ptr()),
                                                          c_strides, optics._c(), float(pixel_size), _stream()))
    return num_out, den_out


class BatchedInsertion:
    """Many reconstructions of uneven box size and particle count inserted
    in one set of launches (rexlib_b200_batched_insert): one persistent
    launch claims the work items of every job. No rexlib operation covers
    it; each job's result is that of one insert_*_slices call on its
    operands (the same bits in the deterministic mode).

    jobs: dicts of numerator, denominator (updated in place), slices,
    transforms, radial_weights, and ctf (kind "ctf") or weights (kind
    "weighted"). The descriptors and the workspace are prepared once, so
    calls are cheap and can be captured in a CUDA graph (after the tuner has
    settled, see rexlib_b200_batched_tuning)."""

    _KINDS = {"plain": _capi.KIND_PLAIN, "ctf": _capi.KIND_CTF, "weighted": _capi.KIND_WEIGHTED}

    def __init__(self, jobs: Sequence[dict], window: GriddingWindow, kind: str = "ctf",
                 optics: CtfOptics | None = None, pixel_size: float = 1.0, *, deterministic: bool | None = None):
        if kind not in self._KINDS:
            raise ValueError(f"kind must be one of {sorted(self._KINDS)}")
        if kind == "ctf" and not isinstance(optics, CtfOptics):
            raise TypeError("the ctf kind needs a CtfOptics")
        self.kind = kind
        self.optics = optics or CtfOptics(300.0, 2.7, 0.1)
        self.pixel_size = float(pixel_size)
        self._keep = []
        self._jobs = (_capi.InsertionJob * len(jobs))()
        for i, job in enumerate(jobs):
            extra_name = {"ctf": "ctf", "weighted": "weights"}.get(kind)
            extra_batches = []
            extra = None
            if extra_name is not None:
                extra = job[extra_name]
                _check_device(extra_name, extra, torch.float32)
                core = 1 if kind == "ctf" else 2
                extra_batches = [_split(extra, core)[0]]
            desc, plan, num_out, den_out, keep = _prepare_insertion(
                job["numerator"], job["denominator"], job["slices"], job["transforms"], job["radial_weights"],
                window, job["numerator"], job["denominator"], deterministic, extra_batches=extra_batches)
            self._keep.extend(keep)
            self._jobs[i].insertion = desc
            if extra is not None:
                e, e_strides = plan.strides(extra, 1 if kind == "ctf" else 2)
                self._keep.append(e)
                self._jobs[i].extra = e.data_ptr()
                self._jobs[i].extra_strides = e_strides
        lib = _capi.load()
        size = ctypes.c_size_t(0)
        _capi.check(lib.rexlib_b200_batched_insertion_workspace_size(self._jobs, len(jobs), self._KINDS[kind],
                                                                     ctypes.byref(size)))
        device = torch.device("cuda", torch.cuda.current_device())
        self.workspace = torch.empty(max(1, size.value), dtype=torch.uint8, device=device)

    def __call__(self) -> None:
        _capi.check(_capi.load().rexlib_b200_batched_insert(
            self._jobs, len(self._jobs), self._KINDS[self.kind], self.optics._c(), self.pixel_size,
            ctypes.c_void_p(self.workspace.data_ptr()), self.workspace.numel(), _stream()))

    def tuning(self) -> tuple[bool, tuple[int, int, int]]:
        """(tuned, (tile cells, shortest run, longest run)) of the job set."""
        tuned = ctypes.c_int32(0)
        config = _capi.TileConfig()
        _capi.check(_capi.load().rexlib_b200_batched_tuning(self._jobs, len(self._jobs), self._KINDS[self.kind],
                                                            ctypes.byref(tuned), ctypes.byref(config)))
        return bool(tuned.value), (config.cells, config.min_hits, config.max_hits)

    def launch_count(self) -> int:
        count = ctypes.c_int32(0)
        _capi.check(_capi.load().rexlib_b200_batched_insertion_launches(self._jobs[0].insertion.mode,
                                                                        ctypes.byref(count)))
        return int(count.value)


def insertion_launch_count(numerator: torch.Tensor, denominator: torch.Tensor, slices: torch.Tensor,
                           transforms: torch.Tensor, radial_weights: torch.Tensor, window: GriddingWindow,
                           deterministic: bool | None = None) -> int:
    """Kernels of this library that an insertion of these operands launches."""
    desc, plan, num_out, den_out, keep = _prepare_insertion(
        numerator, denominator, slices, transforms, radial_weights, window, numerator, denominator, deterministic)
    count = ctypes.c_int32(0)
    _capi.check(_capi.load().rexlib_b200_insertion_launches(ctypes.byref(desc), ctypes.byref(count)))
    return int(count.value)


# --------------------------------------------------------------------------
# Preprocessing


def _resolve_bounds(bounds: float | tuple[float, float]) -> tuple[float, float]:
    if isinstance(bounds, tuple):
        lower, upper = bounds
        return float(lower), float(upper)
    return -float(bounds), float(bounds)


def standardize_background(value: torch.Tensor, key: torch.Tensor, axes: Sequence[int], radius: float,
                           bounds: float | tuple[float, float], context=None, out: torch.Tensor | None = None,
                           *, statistics: torch.Tensor | None = None) -> torch.Tensor:
    """em.standardize_background (python/rexlib/em/_functional.py:30-75):
    standardize the images held in `axes` against the statistics of their
    background (elements farther than `radius` from the centre), replacing
    non-finite or out-of-bounds elements with standard normal draws keyed by
    `key` (uint64, one for all images or broadcast over the batch axes)."""
    _check_device("value", value, torch.float32)
    if not isinstance(key, torch.Tensor) or key.dtype not in (torch.uint64, torch.int64):
        raise TypeError("key must be a uint64 tensor")
    if not key.is_cuda:
        raise ValueError("key must live on a CUDA device")
    lower, upper = _resolve_bounds(bounds)
    if not (radius >= 0.0):
        raise ValueError(f"standardize_background: the radius must be 0 or more, but it is {radius}.")
    if not (lower < 0.0 and upper > 0.0):
        raise ValueError("standardize_background: the bounds must lie on either side of 0, but they are "
                         f"({lower}, {upper}).")
    rank = value.ndim
    axes = [a % rank for a in axes]
    if len(set(axes)) != len(axes):
        raise ValueError("standardize_background: an axis is repeated")
    if len(axes) not in (2, 3):
        raise ValueError("rexlib_b200 standardizes images of 2 or 3 axes")
    batch_axes = [a for a in range(rank) if a not in axes]
    order = batch_axes + list(axes)
    moved = value.permute(*order).contiguous()
    batch_shape = tuple(moved.shape[: len(batch_axes)])
    image_shape = tuple(moved.shape[len(batch_axes):])
    batch = math.prod(batch_shape)
    # Keys broadcast against the batch axes; images sharing a key must be a
    # contiguous run in row-major batch order.
    k = key.reshape((1,) * max(0, len(batch_shape) - key.ndim) + tuple(key.shape)) if key.ndim <= len(
        batch_shape) else key
    if k.ndim != len(batch_shape):
        raise ValueError("the key must have no core axes and broadcast against the batch axes")
    try:
        torch.broadcast_shapes(tuple(k.shape), batch_shape)
    except RuntimeError:
        raise ValueError("the key does not broadcast against the batch axes") from None
    trailing = len(batch_shape)
    while trailing > 0 and k.shape[trailing - 1] == 1:
        trailing -= 1
    if any(k.shape[i] == 1 and batch_shape[i] != 1 for i in range(trailing)):
        raise ValueError("rexlib_b200 needs the images that share a key to be consecutive in the batch order")
    images_per_key = math.prod(batch_shape[trailing:]) if batch_shape else 1
    keys = k.contiguous().reshape(-1)
    identity = order == list(range(rank))
    direct = (out is not None and identity and out.is_cuda and out.dtype == torch.float32 and
              tuple(out.shape) == tuple(value.shape) and out.is_contiguous())
    result = out if direct else torch.empty_like(moved)
    desc = _capi.Standardization()
    desc.result = result.data_ptr()
    desc.value = moved.data_ptr()
    desc.keys = keys.data_ptr()
    desc.images_per_key = max(1, images_per_key)
    desc.batch = batch
    desc.rank = len(image_shape)
    for i, e in enumerate(image_shape):
        desc.extents[i] = e
    desc.radius = float(radius)
    desc.lower_bound = lower
    desc.upper_bound = upper
    if statistics is not None:
        if statistics.dtype != torch.float64 or not statistics.is_cuda or statistics.numel() != 2 * batch:
            raise ValueError("statistics must be a float64 CUDA tensor of batch x 2 elements")
        desc.statistics = statistics.data_ptr()
    _capi.check(_capi.load().rexlib_b200_standardize_background(ctypes.byref(desc), _stream()))
    if direct:
        return out
    inverse = [order.index(i) for i in range(rank)]
    final = result.permute(*inverse)
    if out is not None:
        out.copy_(final)
        return out
    return final if final.is_contiguous() else final.contiguous()


def standardize_background_2d(value, key, radius, bounds, context=None, out=None, *, statistics=None):
    """em.standardize_background_2d: images in the last two axes."""
    return standardize_background(value, key, (-2, -1), radius, bounds, context, out, statistics=statistics)


def standardize_background_3d(value, key, radius, bounds, context=None, out=None, *, statistics=None):
    """em.standardize_background_3d: images in the last three axes."""
    return standardize_background(value, key, (-3, -2, -1), radius, bounds, context, out, statistics=statistics)
