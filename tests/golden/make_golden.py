"""Generate the golden fixtures of this directory.

Run where the reference sources are present (it builds the reference's own
CPU path with oracle/ref/Makefile first):

    python tests/golden/make_golden.py /path/to/rexlib

Writes
- kat.json: the known answers the reference's unit tests hold (Philox4x32-10
  Random123 vectors, tests/unitary/src/backends/cpu/kernels/test_philox.cpp:9-38;
  uniform_open_closed bounds, test_standard_normal.cpp:17-31) plus draws and
  CTF values computed by the reference build for fixed arguments;
- insertion_*.npz: small insertion cases (inputs and the reference outputs,
  float32 and float64) over the windows, variants and parities the
  reference's functor tests cover (test_slice_insertion_functor.cpp:87-117);
- standardize.npz: small standardization cases with the reference outputs.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def rotations(count: int, rng: np.random.Generator) -> np.ndarray:
    """Uniform rotations from normalised Gaussian quaternions."""
    q = rng.standard_normal((count, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


def insertion_case(n: int, big: int, particles: int, volumes: int, kind: str, dtype, seed: int):
    rng = np.random.default_rng(seed)
    h = n // 2 + 1
    H = big // 2 + 1
    cdt = np.complex64 if dtype == np.float32 else np.complex128
    slices = (rng.standard_normal((particles, n, h)) + 1j * rng.standard_normal((particles, n, h))).astype(cdt)
    tr = np.zeros((volumes, particles, 3, 4))
    tr[..., :3] = rotations(volumes * particles, rng).reshape(volumes, particles, 3, 3)
    tr[..., 3] = rng.uniform(-2, 2, (volumes, particles, 3))
    radial = rng.uniform(0.5, 1.5, h)
    radial[-1] = 0.0 if n % 2 == 0 else radial[-1]
    extra = None
    if kind == "ctf":
        e = np.zeros((volumes, particles, 4))
        e[..., 0] = rng.uniform(8000, 25000, (volumes, particles))
        e[..., 1] = e[..., 0] - rng.uniform(0, 800, (volumes, particles))
        e[..., 2] = rng.uniform(0, np.pi, (volumes, particles))
        e[..., 3] = rng.uniform(0, 0.3, (volumes, particles))
        extra = e
    elif kind == "weighted":
        extra = rng.uniform(0, 2, (particles, n, h))
    num = (rng.standard_normal((volumes, big, big, H)) + 1j * rng.standard_normal((volumes, big, big, H)))
    den = rng.uniform(0, 1, (volumes, big, big, H))
    return dict(
        numerator=num.astype(cdt), denominator=den.astype(dtype), slices=slices, transforms=tr.astype(dtype),
        radial=radial.astype(dtype), extra=None if extra is None else extra.astype(dtype))


WINDOWS = {
    "nearest": oracle.Window("nearest", 0.5, 0.0),
    "linear": oracle.Window("linear", 1.0, 0.0),
    "kb15": oracle.Window("kaiser_bessel", 1.5, 6.0),
}
OPTICS = oracle.Optics(300.0, 2.7, 0.1)
PIXEL = 1.3


def main(ref_root: str) -> None:
    if not oracle.build_reference(ref_root):
        raise SystemExit(f"reference sources not found under {ref_root}")
    oracle.build_oracle()

    # Known answers.
    kat = {
        "philox": [
            {"counter": [0, 0, 0, 0], "key": [0, 0], "out": [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]},
            {"counter": [0xffffffff] * 4, "key": [0xffffffff] * 2,
             "out": [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]},
            {"counter": [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], "key": [0xa4093822, 0x299f31d0],
             "out": [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]},
        ],
        "uniform_open_closed": [
            {"bits": 0, "value": 1.0 / 9007199254740992.0},
            {"bits": 1 << 63, "value": 0.5 + 1.0 / 9007199254740992.0},
            {"bits": (1 << 64) - 1, "value": 1.0},
        ],
        "normal_pairs": [],
        "ctf": [],
    }
    for key, block in [(0, 0), (0x0123456789abcdef, 0x100000002), (42, 7), (2**63 + 5, 2**40 + 3)]:
        pair = oracle.standard_normal_pair(key, block, implementation="ref")
        kat["normal_pairs"].append({"key": key, "block": block, "pair": list(pair)})
    for (du, dv, angle, shift, kx, ky, extent) in [
        (15000.0, 14000.0, 0.3, 0.0, 0.0, 0.0, 64), (15000.0, 14000.0, 0.3, 0.0, 12.0, -5.0, 64),
        (25000.0, 8000.0, 2.0, 0.2, 30.0, 0.0, 128), (8000.0, 8000.0, 0.0, 0.0, 0.0, 30.0, 128),
        (20000.0, 19500.0, 1.1, 0.05, 100.0, 77.0, 256),
    ]:
        value = oracle.ctf_f32(OPTICS, PIXEL, extent, du, dv, angle, shift, kx, ky, implementation="ref")
        kat["ctf"].append({"defocus_u": du, "defocus_v": dv, "angle": angle, "phase_shift": shift, "k_x": kx,
                           "k_y": ky, "extent": extent, "value": value})
    kat["ctf_optics"] = {"voltage": OPTICS.voltage, "cs": OPTICS.cs,
                         "amplitude_contrast": OPTICS.amplitude_contrast, "pixel_size": PIXEL}
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1)

    # Insertion cases.
    count = 0
    for dtype, tag in [(np.float32, "f32"), (np.float64, "f64")]:
        arrays = {}
        index = []
        for (n, big) in [(6, 12), (5, 7), (8, 8), (7, 7)]:
            for kind in ["plain", "ctf", "weighted"]:
                for wname, window in WINDOWS.items():
                    volumes = 2 if (n, big) == (8, 8) else 1
                    c = insertion_case(n, big, 4, volumes, kind, dtype, seed=1000 + count)
                    num = c["numerator"].copy()
                    den = c["denominator"].copy()
                    oracle.insert(kind, num, den, c["slices"], c["transforms"], c["radial"], c["extra"],
                                  window=window, optics=OPTICS, pixel_size=PIXEL, implementation="ref", threads=2)
                    name = f"c{count}"
                    for k, v in c.items():
                        if v is not None:
                            arrays[f"{name}_{k}"] = v
                    arrays[f"{name}_out_numerator"] = num
                    arrays[f"{name}_out_denominator"] = den
                    index.append({"name": name, "n": n, "big": big, "kind": kind, "window": wname,
                                  "profile": window.profile, "half_width": window.half_width,
                                  "shape": window.shape})
                    count += 1
        np.savez_compressed(os.path.join(HERE, f"insertion_{tag}.npz"), **arrays)
        with open(os.path.join(HERE, f"insertion_{tag}.json"), "w") as f:
            json.dump({"optics": vars(OPTICS), "pixel_size": PIXEL, "cases": index}, f, indent=1)

    # Standardization cases.
    rng = np.random.default_rng(7)
    arrays = {}
    index = []
    for i, (shape, bounds, shared) in enumerate([
        ((3, 16, 16), (-np.inf, np.inf), False), ((2, 17, 13), (-3.0, 3.0), False),
        ((4, 12, 12), (-2.5, 1.0), True), ((2, 9, 10, 11), (-3.0, 3.0), False),
    ]):
        v = (rng.standard_normal(shape) * rng.uniform(0.5, 3) + rng.uniform(-2, 2)).astype(np.float32)
        v.flat[5] = np.nan
        v.flat[17] = np.inf
        v.flat[40] = 50.0
        keys = (np.array([7], dtype=np.uint64) if shared
                else rng.integers(0, 2**63, shape[0]).astype(np.uint64))
        radius = 0.45 * shape[-1]
        out, stats = oracle.standardize(v, keys, radius, *bounds, image_rank=len(shape) - 1, return_statistics=True,
                                        implementation="ref")
        arrays[f"s{i}_value"] = v
        arrays[f"s{i}_keys"] = keys
        arrays[f"s{i}_out"] = out
        arrays[f"s{i}_stats"] = stats
        index.append({"name": f"s{i}", "radius": radius, "lower": bounds[0], "upper": bounds[1],
                      "rank": len(shape) - 1})
    np.savez_compressed(os.path.join(HERE, "standardize.npz"), **arrays)
    with open(os.path.join(HERE, "standardize.json"), "w") as f:
        json.dump({"cases": index}, f, indent=1)
    print(f"wrote {count} insertion cases and {len(index)} standardization cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/rexlib (the reference source tree)")
    main(sys.argv[1])
