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
           masks: Sequence[torch.Tensor | None] | None = None, error: torch.Tensor | None = None,
           wait_limit_ns: int = 0) -> list:
    """3x3x3 convolution (padding 1) of one volume or two concatenated ones;
    weights (C_out, 27, C_in) BF16, bias FP32. `out` may be two volumes that
    split the output channels (the first takes its channel count). `error`
    (an int32 device tensor) receives a nonzero code when a wait inside the
    kernel ran out; `wait_limit_ns` bounds those waits (0: two seconds)."""
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
    a.wait_limit_ns = int(wait_limit_ns)
    _capi.check(_capi.load().rexlib_b200_conv3d(ctypes.byref(a), _stream()))
    return out


def conv3d_wgrad(inputs: Sequence[torch.Tensor], output_grad: torch.Tensor, weight_grad: torch.Tensor,
                 bias_grad: torch.Tensor | None = None, error: torch.Tensor | None = None,
                 wait_limit_ns: int = 0) -> None:
    """Weight and bias gradients of `conv3d` on the tensor cores, added to
    `weight_grad` ((C_out, 27, C_in) FP32) and `bias_grad` ((C_out,) FP32):
    dw[o, t, i] += sum_v g[v, o] x[v + offset(t), i], db[o] += sum_v g[v, o],
    for the output gradient g (D, H, W, C_out) BF16 and the convolution's
    input volumes (W at least 16). `error` and `wait_limit_ns` as for
    `conv3d`."""
    inputs = list(inputs)
    for i, t in enumerate(inputs):
        _check_volume(f"inputs[{i}]", t)
    _check_volume("output_grad", output_grad)
    D, H, W = inputs[0].shape[:3]
    cout = output_grad.shape[3]
    cin = sum(t.shape[3] for t in inputs)
    if not (weight_grad.is_cuda and weight_grad.dtype == torch.float32 and weight_grad.is_contiguous()
            and tuple(weight_grad.shape) == (cout, 27, cin)):
        raise TypeError("weight_grad must be a contiguous (C_out, 27, C_in) float32 CUDA tensor")
    if bias_grad is not None and not (bias_grad.is_cuda and bias_grad.dtype == torch.float32
                                      and tuple(bias_grad.shape) == (cout,)):
        raise TypeError("bias_grad must be a (C_out,) float32 CUDA tensor")
    a = _capi.Conv3dWgradArgs()
    a.sources = len(inputs)
    for i, t in enumerate(inputs):
        a.inputs[i] = t.data_ptr()
        a.input_channels[i] = t.shape[3]
        a.input_strides[i] = t.stride(2)
    a.depth, a.height, a.width = D, H, W
    a.output_grad = output_grad.data_ptr()
    a.output_channels = cout
    a.output_grad_stride = output_grad.stride(2)
    a.weight_grad = weight_grad.data_ptr()
    a.bias_grad = None if bias_grad is None else bias_grad.data_ptr()
    a.error = None if error is None else error.data_ptr()
    a.wait_limit_ns = int(wait_limit_ns)
    _capi.check(_capi.load().rexlib_b200_conv3d_wgrad(ctypes.byref(a), _stream()))


class UNet:
    """The 3D U-Net prior for cubic volumes of `extent` (16 to 512, a power of
    two): 16-32-64-128 channels, about 1.4 million parameters, residual
    output (input + head). Forward, backward and the Adam step run on the
    library's kernels; the network owns its device buffers."""

    LAYERS = 18

    def __init__(self, extent: int, seed: int = 0):
        self.extent = int(extent)
        handle = ctypes.c_void_p()
        _capi.check(_capi.load().rexlib_b200_unet_create(self.extent, seed, ctypes.byref(handle)))
        self._h = handle
        count = ctypes.c_int64(0)
        _capi.check(_capi.load().rexlib_b200_unet_parameter_count(self._h, ctypes.byref(count)))
        self.parameter_count = int(count.value)
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")

    def close(self) -> None:
        if getattr(self, "_h", None):
            _capi.check(_capi.load().rexlib_b200_unet_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def layer(self, index: int) -> tuple[int, int, tuple[int, int, int, int]]:
        """(weight offset, bias offset, (kind, channels a, channels b, outputs))."""
        wo, bo = ctypes.c_int64(0), ctypes.c_int64(0)
        shape = (ctypes.c_int32 * 4)()
        _capi.check(_capi.load().rexlib_b200_unet_layer(self._h, index, ctypes.byref(wo), ctypes.byref(bo), shape))
        return int(wo.value), int(bo.value), tuple(shape)

    def tensor(self, layer: int, gradient: bool = False) -> torch.Tensor:
        """Layer `layer`'s BF16 output (or its gradient) from the last pass."""
        _, _, (kind, ca, cb, cout) = self.layer(layer)
        level = {0: 0, 1: 0, 2: 1, 3: 1, 4: 2, 5: 2, 6: 3, 7: 3, 8: 2, 9: 2, 10: 2, 11: 1, 12: 1, 13: 1, 14: 0,
                 15: 0, 16: 0}[layer]
        e = self.extent >> level
        out = torch.empty((e, e, e, cout), dtype=torch.bfloat16, device="cuda")
        _capi.check(_capi.load().rexlib_b200_unet_tensor(self._h, 1 if gradient else 0, layer,
                                                         ctypes.c_void_p(out.data_ptr()), _stream()))
        return out

    def parameters(self) -> torch.Tensor:
        out = torch.empty(self.parameter_count, dtype=torch.float32, device="cuda")
        _capi.check(_capi.load().rexlib_b200_unet_copy(self._h, ctypes.c_void_p(out.data_ptr()), None, None, _stream()))
        return out

    def gradients(self) -> torch.Tensor:
        out = torch.empty(self.parameter_count, dtype=torch.float32, device="cuda")
        _capi.check(_capi.load().rexlib_b200_unet_copy(self._h, None, ctypes.c_void_p(out.data_ptr()), None, _stream()))
        return out

    def load(self, parameters: torch.Tensor) -> None:
        p = parameters.to(device="cuda", dtype=torch.float32).contiguous()
        if p.numel() != self.parameter_count:
            raise ValueError("the parameter vector does not fit this network")
        _capi.check(_capi.load().rexlib_b200_unet_copy(self._h, None, None, ctypes.c_void_p(p.data_ptr()), _stream()))
        torch.cuda.current_stream().synchronize()

    def _volume(self, name, t):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
                and tuple(t.shape) == (self.extent,) * 3):
            raise ValueError(f"{name} must be a contiguous float32 CUDA volume of extent {self.extent}")

    def forward(self, x: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        self._volume("input", x)
        out = torch.empty_like(x) if out is None else out
        self._volume("output", out)
        # The network reads both again in backward: hold them until then.
        self._input, self._output = x, out
        _capi.check(_capi.load().rexlib_b200_unet_forward(self._h, ctypes.c_void_p(x.data_ptr()),
                                                          ctypes.c_void_p(out.data_ptr()), _stream()))
        return out

    def backward(self, target: torch.Tensor) -> torch.Tensor:
        """Adds the gradients of 0.5 mean (output - target)^2; returns the loss
        (a device scalar, accumulated since the last step)."""
        self._volume("target", target)
        _capi.check(_capi.load().rexlib_b200_unet_backward(self._h, ctypes.c_void_p(target.data_ptr()),
                                                           ctypes.c_void_p(self.loss.data_ptr()), _stream()))
        return self.loss

    def step(self, learning_rate: float) -> None:
        _capi.check(_capi.load().rexlib_b200_unet_adam_step(self._h, float(learning_rate), _stream()))
        self.loss.zero_()

    def error(self) -> int:
        code = ctypes.c_int32(0)
        _capi.check(_capi.load().rexlib_b200_unet_error(self._h, ctypes.byref(code)))
        return int(code.value)


# --------------------------------------------------------------------------
# Volumes, phantoms and the reconstruction loop

import math  # noqa: E402

import numpy as np  # noqa: E402

from . import em, fourier  # noqa: E402


def rfft3(volume: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """Unnormalised R2C of a (N, N, N) float32 volume, N in {32, 64, 128, 256}."""
    n = volume.shape[0]
    if out is None:
        out = torch.empty((n, n, n // 2 + 1), dtype=torch.complex64, device=volume.device)
    _capi.check(_capi.load().rexlib_b200_rfft3(ctypes.c_void_p(out.data_ptr()),
                                               ctypes.c_void_p(volume.contiguous().data_ptr()), n, _stream()))
    return out


def fsc(a: torch.Tensor, b: torch.Tensor) -> np.ndarray:
    """Fourier shell correlation of two half spectra, shells 0 .. N/2."""
    n = a.shape[0]
    sums = torch.empty(3 * (n // 2 + 1), dtype=torch.float64, device=a.device)
    _capi.check(_capi.load().rexlib_b200_fsc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), n,
                                             ctypes.c_void_p(sums.data_ptr()), _stream()))
    s = sums.cpu().numpy().reshape(3, -1)
    return s[0] / np.sqrt(np.maximum(s[1] * s[2], 1e-300))


def resolution_shell(curve: np.ndarray, threshold: float = 0.143) -> float:
    """The shell where the correlation first falls below `threshold`
    (linearly interpolated between shells; the last shell if it never does).
    The resolution is N * pixel / shell."""
    for s in range(1, len(curve)):
        if curve[s] < threshold:
            lo, hi = curve[s - 1], curve[s]
            return float(s - 1 + (lo - threshold) / (lo - hi)) if lo != hi else float(s)
    return float(len(curve) - 1)


def blob_phantom(rng: np.random.Generator, extent: int, count: int, kind: str = "blobs",
                 scale: float | None = None, sigma: tuple[float, float] | None = None) -> np.ndarray:
    """Blobs (amplitude, sigma, centre x, y, z from the volume centre), float32
    (count, 5): Gaussian blobs in a sphere of radius 0.375 N (sigma uniform in
    `sigma` voxels, by default 2-4 voxels times `scale`, itself by default
    N / 64), or a helical filament of blobs (sigma 1.5-2.5 times `scale`, or
    in the lower half of `sigma`)."""
    scale = extent / 64.0 if scale is None else scale
    lo, hi = (2.0 * scale, 4.0 * scale) if sigma is None else sigma
    b = np.zeros((count, 5), np.float32)
    b[:, 0] = rng.uniform(0.5, 1.5, count)
    b[:, 1] = rng.uniform(lo, hi, count)
    if kind == "helix":
        t = np.linspace(0, 1, count)
        turns, radius, length = rng.uniform(2, 4), rng.uniform(0.1, 0.2) * extent, 0.6 * extent
        phase = rng.uniform(0, 2 * np.pi)
        b[:, 2] = radius * np.cos(2 * np.pi * turns * t + phase)
        b[:, 3] = radius * np.sin(2 * np.pi * turns * t + phase)
        b[:, 4] = (t - 0.5) * length
        b[:, 1] = rng.uniform(0.75 * lo, 0.625 * (lo + hi) if sigma is not None else 1.25 * lo, count)
    else:
        d = rng.standard_normal((count, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        r = 0.375 * extent * rng.uniform(0, 1, count) ** (1 / 3)
        b[:, 2:] = d * r[:, None]
    return b


def random_orientations(count: int, rng: np.random.Generator) -> np.ndarray:
    """Transforms (count, 3, 4): uniform rotations (normalised Gaussian
    quaternions), no shift."""
    q = rng.standard_normal((count, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    r = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], -2)
    t = np.zeros((count, 3, 4), np.float32)
    t[:, :, :3] = r
    return t


OPTICS = em.CtfOptics(300.0, 2.7, 0.1)


def _slices(blobs_d, n, tr_d, ctf_d, noise, seed):
    out = torch.empty((tr_d.shape[0], n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    _capi.check(_capi.load().rexlib_b200_phantom_slices(
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(blobs_d.data_ptr()), blobs_d.shape[0], tr_d.shape[0], n,
        ctypes.c_void_p(tr_d.data_ptr()), ctypes.c_void_p(ctf_d.data_ptr()), OPTICS._c(), 1.0, float(noise), seed,
        _stream()))
    return out


def blob_spectrum(blobs: np.ndarray, extent: int, cutoff: float = -1.0) -> torch.Tensor:
    b = torch.from_numpy(np.ascontiguousarray(blobs, np.float32)).cuda()
    out = torch.empty((extent, extent, extent // 2 + 1), dtype=torch.complex64, device="cuda")
    _capi.check(_capi.load().rexlib_b200_blob_spectrum(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                                       b.shape[0], extent, float(cutoff), _stream()))
    return out


class Dataset:
    """Noisy CTF-modulated particles of a blob phantom at a given SNR (signal
    variance over noise variance of the images), inserted into the
    accumulators of an extent-N reconstruction (N = n)."""

    def __init__(self, blobs: np.ndarray, extent: int, particles: int, snr: float, seed: int, chunk: int = 4096):
        rng = np.random.default_rng(seed)
        n = extent
        h = n // 2 + 1
        self.extent = n
        self.blobs = blobs
        blobs_d = torch.from_numpy(np.ascontiguousarray(blobs, np.float32)).cuda()
        tr = random_orientations(particles, rng)
        ctf = np.stack([rng.uniform(8000, 25000, particles), rng.uniform(8000, 25000, particles),
                        rng.uniform(0, np.pi, particles), np.zeros(particles)], -1).astype(np.float32)
        tr_d, ctf_d = torch.from_numpy(tr).cuda(), torch.from_numpy(ctf).cuda()
        # Image variance of the noiseless data (Parseval over the half spectrum).
        probe = _slices(blobs_d, n, tr_d[:64], ctf_d[:64], 0.0, 0)
        power = probe.abs() ** 2
        full = power[:, :, 0].sum(1) + 2 * power[:, :, 1:h - 1].sum((1, 2)) + power[:, :, h - 1].sum(1)
        var = (full - power[:, 0, 0]) / float(n) ** 4
        signal_var = float(var.mean())
        self.noise = math.sqrt(n * n * signal_var / snr / 2.0)
        self.num = torch.zeros((n, n, h), dtype=torch.complex64, device="cuda")
        self.den = torch.zeros((n, n, h), dtype=torch.float32, device="cuda")
        radial = torch.ones(h, dtype=torch.float32, device="cuda")
        self._parts = []
        for start in range(0, particles, chunk):
            stop = min(particles, start + chunk)
            sl = _slices(blobs_d, n, tr_d[start:stop], ctf_d[start:stop], self.noise, seed * 1000003 + start)
            em.insert_ctf_slices(self.num, self.den, sl, tr_d[start:stop], ctf_d[start:stop], radial,
                                 em.GriddingWindow.linear(), OPTICS, 1.0, numerator_out=self.num,
                                 denominator_out=self.den)

    def wiener(self, constant: float = 1e-3) -> torch.Tensor:
        return fourier.wiener_irfft3(self.num, self.den, constant)

    def truth(self, cutoff: float = -1.0) -> torch.Tensor:
        """The phantom itself, band-limited at `cutoff` (shells)."""
        return fourier.irfft3(blob_spectrum(self.blobs, self.extent, cutoff))

    def resolution(self, volume: torch.Tensor) -> tuple[float, np.ndarray]:
        """FSC-0.143 shell of `volume` against the phantom, and the curve."""
        curve = fsc(rfft3(volume), blob_spectrum(self.blobs, self.extent))
        return resolution_shell(curve), curve


def regularised_step(net: UNet, numerator: torch.Tensor, denominator: torch.Tensor, x: torch.Tensor,
                     weight: float) -> torch.Tensor:
    """One iteration of the prior-regularised reconstruction:
    irfft3((N + c F(U(x))) / (D + c)), U the network, N and D the
    accumulators, c the prior's weight."""
    extent = numerator.shape[0]
    p = rfft3(net.forward(x))
    combined = torch.empty_like(numerator)
    _capi.check(_capi.load().rexlib_b200_prior_wiener(
        ctypes.c_void_p(combined.data_ptr()), ctypes.c_void_p(numerator.data_ptr()),
        ctypes.c_void_p(denominator.data_ptr()), ctypes.c_void_p(p.data_ptr()), extent, float(weight), _stream()))
    return fourier.irfft3(combined)


def regularised(net: UNet, data: Dataset, iterations: int = 10, weight: float | None = None,
                constant: float = 1e-3) -> torch.Tensor:
    """Reconstruction with the learned prior as the regulariser: from the
    Wiener map, `iterations` times x <- irfft3((N + c F(U(x))) / (D + c)),
    U the network, N and D the accumulators; c defaults to the mean of D."""
    if net.extent != data.extent:
        raise ValueError("the network and the reconstruction must have one extent")
    c = float(data.den.mean()) if weight is None else float(weight)
    x = data.wiener(constant)
    for _ in range(iterations):
        x = regularised_step(net, data.num, data.den, x, c)
    return x


def make_pairs(count: int, extent: int, seed: int, particles=(2000, 20000), snr=(0.05, 0.2),
               blobs=(20, 40), sigma: tuple[float, float] | None = None, accumulators: bool = False):
    """Training pairs generated on the GPU: the Wiener reconstruction
    (constant 1e-3) of a seeded blob or helical-filament phantom (blob widths
    from `sigma` voxels, by default blob_phantom's) from a random number of
    noisy particles at a random SNR, and the phantom low-passed to half the
    Nyquist frequency. Returns (inputs, targets), each (count, N, N, N)
    float32, and with `accumulators` also each pair's insertion
    accumulators (numerators, denominators), for training on the prior's
    own iterates."""
    rng = np.random.default_rng(seed)
    inputs = torch.empty((count, extent, extent, extent), dtype=torch.float32, device="cuda")
    targets = torch.empty_like(inputs)
    numerators, denominators = [], []
    for i in range(count):
        kind = "helix" if i % 4 == 3 else "blobs"
        b = blob_phantom(rng, extent, int(rng.integers(blobs[0], blobs[1] + 1)), kind, sigma=sigma)
        p = int(rng.integers(particles[0], particles[1] + 1))
        s = float(rng.uniform(*snr))
        data = Dataset(b, extent, p, s, seed=int(rng.integers(1, 2**31)))
        inputs[i] = data.wiener()
        targets[i] = data.truth(cutoff=extent / 4.0)
        if accumulators:
            numerators.append(data.num)
            denominators.append(data.den)
    if accumulators:
        return inputs, targets, numerators, denominators
    return inputs, targets


def train(net: UNet, inputs: torch.Tensor, targets: torch.Tensor, steps: int, learning_rate: float = 1e-3,
          seed: int = 0) -> list[float]:
    """Adam steps, one pair a step in a seeded random order; the losses."""
    order = np.random.default_rng(seed).integers(0, inputs.shape[0], steps)
    losses = []
    loss = None
    for k, i in enumerate(order):
        net.forward(inputs[i])
        loss = net.backward(targets[i])
        if k % 50 == 49 or k == steps - 1:
            losses.append(float(loss.item()))
        net.step(learning_rate)
    return losses


def train_on_iterates(net: UNet, inputs: torch.Tensor, targets: torch.Tensor, numerators: list,
                      denominators: list, steps: int, weight_factor: float = 6.0, max_iterations: int = 6,
                      learning_rate: float = 1e-3, final_rate: float = 1e-4, seed: int = 1,
                      average_from: float = 1.0) -> list[float]:
    """Adam steps that also show the network its own iterates: every other
    step the input is not the pair's Wiener map but the result of 1 to
    `max_iterations` regularised iterations with the current network (prior
    weight `weight_factor` times the mean of the pair's denominator), so that
    the network stays accurate along the iteration it is used in. The rate
    falls from `learning_rate` to `final_rate` on a cosine.

    With `average_from` below 1, the network ends with the mean of its
    parameters taken every 5 steps from that fraction of the steps on (the
    weights of the last steps averaged, which evens out where single Adam
    steps leave them)."""
    rng = np.random.default_rng(seed)
    order = rng.integers(0, inputs.shape[0], steps)
    losses = []
    average = None
    snapshots = 0
    for k, i in enumerate(order):
        x = inputs[i]
        if k % 2 == 1:
            c = weight_factor * float(denominators[i].mean())
            for _ in range(int(rng.integers(1, max_iterations + 1))):
                x = regularised_step(net, numerators[i], denominators[i], x, c)
            x = x.contiguous()
        net.forward(x)
        loss = net.backward(targets[i])
        if k % 50 == 49 or k == steps - 1:
            losses.append(float(loss.item()))
        rate = final_rate + 0.5 * (learning_rate - final_rate) * (1.0 + math.cos(math.pi * k / max(1, steps)))
        net.step(rate)
        if k >= average_from * steps and (steps - 1 - k) % 5 == 0:
            snapshot = net.parameters()
            average = snapshot if average is None else average.add_(snapshot)
            snapshots += 1
    if snapshots > 0:
        net.load(average / snapshots)
    return losses


def conv_flops(extent: int) -> float:
    """Multiply-add FLOPs (2 per MAC) of one forward pass: the 3x3x3
    convolutions and the transposed convolutions."""
    total = 0.0
    levels = {0: extent ** 3, 1: (extent // 2) ** 3, 2: (extent // 4) ** 3, 3: (extent // 8) ** 3}
    convs = [(0, 1, 16), (0, 16, 16), (1, 16, 32), (1, 32, 32), (2, 32, 64), (2, 64, 64), (3, 64, 128), (3, 128, 128),
             (2, 128, 64), (2, 64, 64), (1, 64, 32), (1, 32, 32), (0, 32, 16), (0, 16, 16)]
    for lvl, cin, cout in convs:
        total += 2.0 * 27 * cin * cout * levels[lvl]
    for lvl, cin, cout in [(3, 128, 64), (2, 64, 32), (1, 32, 16)]:
        total += 2.0 * 8 * cin * cout * levels[lvl]
    return total
