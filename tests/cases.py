"""Seeded synthetic inputs shared by the tests (numpy, host side)."""

from __future__ import annotations

import numpy as np


def rotations(count: int, rng: np.random.Generator) -> np.ndarray:
    """Uniform random rotations (normalised Gaussian quaternions)."""
    q = rng.standard_normal((count, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


def insertion_inputs(n: int, big: int, particles: int, volumes: int = 1, kind: str = "plain", seed: int = 0,
                     per_volume_slices: bool = False, radial_per_particle: bool = False,
                     shift: float = 2.0, zero_accumulators: bool = False):
    """float32 inputs: slices (P,n,h) or (V,P,n,h), transforms (V,P,3,4),
    radial (h) or (P,h), extra (ctf (V,P,4) or weights (P,n,h)), accumulators."""
    rng = np.random.default_rng(seed)
    h = n // 2 + 1
    H = big // 2 + 1
    shape = (volumes, particles, n, h) if per_volume_slices else (particles, n, h)
    slices = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    tr = np.zeros((volumes, particles, 3, 4))
    tr[..., :3] = rotations(volumes * particles, rng).reshape(volumes, particles, 3, 3)
    tr[..., 3] = rng.uniform(-shift, shift, (volumes, particles, 3))
    radial = rng.uniform(0.5, 1.5, (particles, h) if radial_per_particle else (h,)).astype(np.float32)
    extra = None
    if kind == "ctf":
        e = np.zeros((volumes, particles, 4))
        e[..., 0] = rng.uniform(8000, 25000, (volumes, particles))
        e[..., 1] = e[..., 0] - rng.uniform(0, 800, (volumes, particles))
        e[..., 2] = rng.uniform(0, np.pi, (volumes, particles))
        e[..., 3] = rng.uniform(0, 0.3, (volumes, particles))
        extra = e.astype(np.float32)
    elif kind == "weighted":
        extra = rng.uniform(0, 2, (particles, n, h)).astype(np.float32)
    if zero_accumulators:
        num = np.zeros((volumes, big, big, H), np.complex64)
        den = np.zeros((volumes, big, big, H), np.float32)
    else:
        num = (rng.standard_normal((volumes, big, big, H)) + 1j * rng.standard_normal((volumes, big, big, H))
               ).astype(np.complex64)
        den = rng.uniform(0, 1, (volumes, big, big, H)).astype(np.float32)
    return dict(numerator=num, denominator=den, slices=slices, transforms=tr.astype(np.float32), radial=radial,
                extra=extra)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    d = np.linalg.norm((a - b).ravel())
    s = np.linalg.norm(b.ravel())
    return float(d / s) if s > 0 else float(d)
