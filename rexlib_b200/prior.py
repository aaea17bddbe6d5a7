"""The learned prior: a 3D U-Net that regularises the reconstruction.

Volumes are channels-last BF16 torch tensors (D, H, W, C) on the GPU; every
operation is a kernel of librexlib_b200.so reached through its C-ABI (the
3x3x3 convolutions on the tcgen05 tensor cores). No counterpart in the
reference: rexlib has no learned component.
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence

import torch

from . import _capi

EPILOGUE_NONE = 0
EPILOGUE_RELU = 1
EPILOGUE_MASK = 2


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check_volume(name: str, t: torch.Tensor) -> None:
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.bfloat16 and t.ndim == 4):
        raise TypeError(f"{name} must be a (D, H, W, C) bfloat16 CUDA tensor")
    if t.stride(3) != 1 or t.stride(1) != t.stride(2) * t.shape[2] or t.stride(0) != t.stride(1) * t.shape[1]:
        raise ValueError(f"{name} must hold its voxels at one stride, channels contiguous")


def conv3d(inputs: Sequence[torch.Tensor], weights: torch.Tensor, bias: torch.Tensor | None = None,
           epilogue: int = EPILOGUE_NONE, out: Sequence[torch.Tensor] | torch.Tensor | None = None,
           masks: Sequence[torch.Tensor | None] | None = None, error: torch.Tensor | None = None) -> list:
    """3x3x3 convolution (padding 1) of one volume or two concatenated ones;
    weights (C_out, 27, C_in) BF16, bias FP32. `out` may be two volumes that
    split the output channels (the first takes its channel count)."""
    inputs = list(inputs)
    for i, t in enumerate(inputs):
        _check_volume(f"inputs[{i}]", t)
    D, H, W = inputs[0].shape[:3]
    cout = weights.shape[0]
    if out is None:
        out = [torch.empty((D, H, W, cout), dtype=torch.bfloat16, device=inputs[0].device)]
    elif isinstance(out, torch.Tensor):
        out = [out]
    out = list(out)
    a = _capi.Conv3dArgs()
    a.sources = len(inputs)
    for i, t in enumerate(inputs):
        a.inputs[i] = t.data_ptr()
        a.input_channels[i] = t.shape[3]
        a.input_strides[i] = t.stride(2)
    a.depth, a.height, a.width = D, H, W
    a.weights = weights.contiguous().data_ptr()
    a.bias = None if bias is None else bias.data_ptr()
    a.output_channels = cout
    a.epilogue = epilogue
    for i, t in enumerate(out):
        _check_volume(f"out[{i}]", t)
        a.outputs[i] = t.data_ptr()
        a.output_strides[i] = t.stride(2)
    a.output_split = out[0].shape[3] if len(out) == 2 else 0
    if masks is not None:
        for i, m in enumerate(masks):
            if m is not None:
                _check_volume(f"masks[{i}]", m)
                a.masks[i] = m.data_ptr()
                a.mask_strides[i] = m.stride(2)
    a.error = None if error is None else error.data_ptr()
    _capi.check(_capi.load().rexlib_b200_conv3d(ctypes.byref(a), _stream()))
    return out
