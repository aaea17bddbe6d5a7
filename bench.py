"""Benchmark: CTF-weighted trilinear Fourier-slice insertion at a 256^2 box.

Workload (the headline configuration): 100,000 particles of 256 x 256
(half spectra 256 x 129 complex64, 26.4 GB resident in HBM) inserted with
their CTF (300 kV, Cs 2.7 mm, Q 0.1, 1.0 A/px, defocus U/V uniform
0.8-2.5 um, astigmatism angle uniform 0-180 deg) at uniform random SO(3)
orientations into a 256^3 complex64 numerator and float32 denominator,
throughput mode. A step zeroes the accumulators and inserts every particle.
Inputs (26.4 GB) exceed the L2 (126 MB), so no flush is needed.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line on rank 0. Under torchrun each rank runs an independent replica
of the workload: the path has no exchange step (the accumulators of several
GPUs would be summed once, after all insertions), so the replicas measure
weak scaling with the time of the slowest rank.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particles/s inserted (256^2 box)"
UNIT = "particles/s"
PIXEL_SIZE = 1.0
OPTICS = (300.0, 2.7, 0.1)
# Gridding windows: (oracle profile name, half-width, Kaiser-Bessel shape, name in the workload).
WINDOWS = {
    "nearest": ("nearest", 0.5, 0.0, "nearest"),
    "linear": ("linear", 1.0, 0.0, "trilinear"),
    "kb15": ("kaiser_bessel", 1.5, 6.0, "Kaiser-Bessel w 1.5"),
    "kb2": ("kaiser_bessel", 2.0, 9.0, "Kaiser-Bessel w 2"),
}


def gpu_window(em, name: str):
    profile, width, shape, _ = WINDOWS[name]
    if profile == "nearest":
        return em.GriddingWindow.nearest()
    if profile == "linear":
        return em.GriddingWindow.linear()
    return em.GriddingWindow.kaiser_bessel(width, shape)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=None,
                   help="timed steps (default 5; 4000 for the wiener workload, one volume a step, and 2000 for "
                        "the arrays workload, so the clock sampler sees the timed region)")
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--particles", type=int, default=100_000)
    p.add_argument("--box", type=int, default=256)
    p.add_argument("--mode", default="throughput", choices=["throughput", "deterministic"])
    p.add_argument("--window", default="linear", choices=sorted(WINDOWS),
                   help="gridding window of the insertion (linear: the headline)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--precision", default="f32", choices=["f32", "f64"],
                   help="insertion: the operands' element type (f64: complex128 slices and accumulators; no e2e or "
                        "CPU legs)")
    p.add_argument("--workload", default="insertion",
                   choices=["insertion", "frontend", "wiener", "pipeline", "arrays", "batched", "prior", "conv3d",
                            "unet"],
                   help="insertion: the headline; frontend: standardize + R2C with the CTF epilogue "
                        "(1,000,000 images of 128^2, in chunks); wiener: the Wiener divide + irfft3 at 256^3; "
                        "pipeline: standardize, R2C, CTF insertion and the Wiener C2R of --particles images "
                        "of --box^2; arrays: divide, add and fill of complex64 arrays of 2^26 elements; batched: 48 "
                        "ragged CTF reconstructions in one batched call against one call per job")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="insertion: skip the other configurations' records (the other mode, front end, 64^3 "
                        "pipeline, Wiener C2R)")
    p.add_argument("--images", type=int, default=1_000_000, help="frontend: images a step")
    p.add_argument("--chunk", type=int, default=100_000, help="frontend: images a call")
    p.add_argument("--image-box", type=int, default=128, help="frontend: image extent (128: the configured front end)")
    p.add_argument("--frontend-path", default=None, choices=["fused", "separate"],
                   help="frontend and pipeline: one fused standardization + R2C kernel (the default at 64^2, "
                        "128^2 and 256^2), or the two calls (the default otherwise)")
    p.add_argument("--prior-extent", type=int, default=128, help="prior: volume extent of the training pairs")
    p.add_argument("--pairs", type=int, default=2000, help="prior: training pairs")
    p.add_argument("--train-steps", type=int, default=1000, help="prior: Adam steps on the Wiener maps")
    p.add_argument("--iterate-steps", type=int, default=1000,
                   help="prior: further Adam steps, every other one on the network's own regularised iterates")
    p.add_argument("--iterate-depth", type=int, default=10,
                   help="prior: the most regularised iterations behind one of those inputs")
    p.add_argument("--eval-extent", type=int, default=256, help="prior: extent of the regularised reconstruction")
    p.add_argument("--eval-particles", type=int, default=40000,
                   help="prior: particles of the evaluation (all of them; half for the 50%% case)")
    p.add_argument("--eval-blobs", type=int, default=200, help="prior: blobs of the evaluation phantom")
    p.add_argument("--conv-channels", default="64,64",
                   help="conv3d: input and output channels of the convolution (at --prior-extent)")
    p.add_argument("--average-from", type=float, default=0.6,
                   help="prior: average the network's parameters over the iterate steps from this fraction on "
                        "(1: keep the last step's)")
    p.add_argument("--train", action="store_true", help="unet: time training steps (forward, backward, Adam)")
    p.add_argument("--conv-pass", default="forward", choices=["forward", "wgrad"],
                   help="conv3d: the convolution, or its weight and bias gradients")
    args = p.parse_args()
    if args.steps is None:
        args.steps = {"wiener": 4000, "arrays": 2000}.get(args.workload, 5)
    return args


def bytes_per_particle(n: int, big: int, particles: int, real_bytes: int = 4) -> float:
    """Algorithmic bytes per particle: the half spectrum read once, its
    transform and CTF, and one read + write of both accumulators amortised
    (elements of real_bytes: 4 for float32, 8 for float64)."""
    h = n // 2 + 1
    H = big // 2 + 1
    return real_bytes * (n * h * 2 + 12 + 4 + 2.0 * big * big * H * 3 / particles)


def measured_peak() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def rotations(count: int, rng: np.random.Generator) -> np.ndarray:
    q = rng.standard_normal((count, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


def host_parameters(particles: int, seed: int):
    """Transforms (P, 3, 4) and CTF parameters (P, 4), float32."""
    rng = np.random.default_rng(seed)
    tr = np.zeros((particles, 3, 4), np.float64)
    tr[:, :, :3] = rotations(particles, rng)
    tr[:, :2, 3] = rng.uniform(-2.0, 2.0, (particles, 2))
    ctf = np.zeros((particles, 4), np.float64)
    ctf[:, 0] = rng.uniform(8000.0, 25000.0, particles)
    ctf[:, 1] = rng.uniform(8000.0, 25000.0, particles)
    ctf[:, 2] = rng.uniform(0.0, np.pi, particles)
    return tr.astype(np.float32), ctf.astype(np.float32)


def synth_slices(torch, particles: int, n: int, device, seed: int, chunk: int = 4096):
    """Seeded complex64 half spectra (P, n, h) on the device: per particle a
    band-limited signal (a Gaussian envelope) under complex Gaussian noise at
    an SNR of 0.1, built chunk by chunk on the device."""
    h = n // 2 + 1
    out = torch.empty((particles, n, h), dtype=torch.complex64, device=device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    ky = torch.fft.fftfreq(n, device=device)[:, None]
    kx = torch.fft.rfftfreq(n, device=device)[None, :]
    envelope = torch.exp(-(kx * kx + ky * ky) * (2 * math.pi ** 2 * 4.0))
    signal_power = float((envelope ** 2).mean())
    noise_sigma = math.sqrt(signal_power / 0.1 / 2)
    for start in range(0, particles, chunk):
        stop = min(particles, start + chunk)
        m = stop - start
        phase = torch.rand((m, 1, 1), generator=g, device=device) * 2 * math.pi
        sig = envelope[None] * torch.polar(torch.ones_like(phase), phase)
        noise = torch.randn((m, n, h, 2), generator=g, device=device) * noise_sigma
        out[start:stop] = sig + torch.view_as_complex(noise)
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to start: the timed region begins once it samples.
            deadline = time.perf_counter() + 3.0
            while not self.lines and time.perf_counter() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
            self.lines.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sms)), "sm_max_mhz": max(maxes), "reasons": sorted(reasons),
                "samples": len(sms)}


# --------------------------------------------------------------------------
# Reference CPU arm


def reference_sample(particles_total: int, n: int, big: int, seed: int, budget_s: float, threads: int,
                     window: str = "linear"):
    """Time the reference's own CPU insertion (oracle/_ref/libref.so, the
    reference sources compiled as they are) on a bounded sample of the
    workload: calls of a pool of particles with the workload's box, CTF and
    orientation distributions, repeated until `budget_s` seconds have run.
    Returns (particles/s, sample particles, seconds, kind)."""
    import oracle

    kind = "reference" if oracle.ref(strict=False) is not None else "port"
    h = n // 2 + 1
    H = big // 2 + 1
    rng = np.random.default_rng(seed)
    pool = 512
    tr, ctf = host_parameters(pool, seed)
    radial = np.ones(h, np.float32)
    num = np.zeros((1, big, big, H), np.complex64)
    den = np.zeros((1, big, big, H), np.float32)
    sl = (rng.standard_normal((pool, n, h)) + 1j * rng.standard_normal((pool, n, h))).astype(np.complex64)

    def run(count):
        start = time.perf_counter()
        oracle.insert("ctf", num, den, sl[:count], tr[None, :count], radial, ctf[None, :count],
                      window=oracle.Window(*WINDOWS[window][:3]), optics=oracle.Optics(*OPTICS), pixel_size=PIXEL_SIZE,
                      implementation="ref_fast" if kind == "reference" else "oracle", threads=threads)
        return time.perf_counter() - start

    run(min(pool, 32))  # warm the pool and the caches
    done, elapsed = 0, 0.0
    while elapsed < budget_s and done < particles_total:
        count = min(pool, particles_total - done)
        elapsed += run(count)
        done += count
    return done / elapsed, done, elapsed, kind


def insertion_config(args, world: int) -> dict:
    """The insertion workload's `config`, the same on both arms."""
    P, n = args.particles, args.box
    f64 = getattr(args, "precision", "f32") == "f64"
    return {"workload": f"insert_ctf_slices {P} x {n}^2 into {n}^3, {WINDOWS[args.window][3]}, {args.mode}" +
                        (", float64" if f64 else ""),
            "particles": P, "box": n, "volume": n, "mode": args.mode, "window": args.window,
            "parallelism": f"replicas{world}", "l2": "inputs 26.4 GB > L2, no flush" if n == 256 and P == 100_000
            else f"inputs {P * n * (n // 2 + 1) * 8 / 1e9:.1f} GB, no flush"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    seconds_per_step = max(5.0, 60.0 / max(1, args.steps + args.warmup))
    values = []
    last = None
    for step in range(args.warmup + args.steps):
        rate, count, elapsed, kind = reference_sample(args.particles, args.box, args.box, 100 + step,
                                                     seconds_per_step, threads, args.window)
        last = (count, elapsed, kind)
        if step >= args.warmup:
            values.append(rate)
    value = float(np.median(values))
    count, elapsed, kind = last
    sample = (f"{count} of {args.particles} particles per step ({args.box}^2 box, CTF, {WINDOWS[args.window][3]}, "
              f"into {args.box}^3), {threads} threads; the reference's CPU functor, which sums in its own fixed "
              f"order whatever the mode")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * count / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": insertion_config(args, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# Our arm


def run_frontend(args):
    """Standardization + R2C with the CTF epilogue over 1,000,000 images of
    128^2 (pure noise, mean U[-2,2], sigma U[0.5,3]), radius 0.45 n, defocus
    U[0.5,4] um, 200/300 kV 50/50, in chunks of 100,000 images. The fused
    path (the default at 64 and 128) runs both in one kernel; the separate
    path runs the standardization and then the R2C. One JSON line."""
    import torch

    from rexlib_b200 import em, fourier

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    n, total, chunk = args.image_box, args.images, args.chunk
    if total % chunk:
        raise SystemExit("--images must be a multiple of --chunk")
    if args.frontend_path is None:
        args.frontend_path = "fused" if n in (64, 128, 256) else "separate"
    fused = args.frontend_path == "fused"
    if fused and n not in (64, 128, 256):
        raise SystemExit("the fused front end runs 64^2, 128^2 and 256^2 images: use --frontend-path separate")
    g = torch.Generator(device=device)
    g.manual_seed(7)
    images = torch.empty((chunk, n, n), dtype=torch.float32, device=device)
    images.normal_(generator=g)
    images.mul_(torch.rand((chunk, 1, 1), generator=g, device=device) * 2.5 + 0.5)
    images.add_(torch.rand((chunk, 1, 1), generator=g, device=device) * 4 - 2)
    keys = torch.arange(1, chunk + 1, dtype=torch.int64, device=device)
    rng = np.random.default_rng(8)
    ctf = torch.from_numpy(np.stack([rng.uniform(5000, 40000, chunk), rng.uniform(5000, 40000, chunk),
                                     rng.uniform(0, np.pi, chunk), np.zeros(chunk)], -1).astype(np.float32)).to(device)
    volts = torch.from_numpy(np.where(rng.uniform(0, 1, chunk) < 0.5, 200.0, 300.0).astype(np.float32)).to(device)
    optics = em.CtfOptics(300.0, 2.7, 0.1)
    std = None if fused else torch.empty_like(images)
    stream = torch.cuda.current_stream()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    phase_ms = [0.0, 0.0]

    def chunk_call(timed):
        if timed:
            e0.record(stream)
        if fused:
            fourier.standardize_rfft2_ctf(images, keys, 0.45 * n, (-np.inf, np.inf), ctf, optics, 1.0, voltage=volts,
                                          weights=False)
            if timed:
                e1.record(stream)
                e2.record(stream)
        else:
            em.standardize_background_2d(images, keys, 0.45 * n, (-np.inf, np.inf), out=std)
            if timed:
                e1.record(stream)
            fourier.rfft2_ctf(std, ctf, optics, 1.0, voltage=volts, weights=False)
            if timed:
                e2.record(stream)
        if timed:
            e2.synchronize()
            phase_ms[0] += e0.elapsed_time(e1)
            phase_ms[1] += e1.elapsed_time(e2)

    for _ in range(args.warmup):
        for _ in range(total // chunk):
            chunk_call(False)
    torch.cuda.synchronize()
    with ClockSampler(0) as clocks:
        begin = torch.cuda.Event(enable_timing=True)
        finish = torch.cuda.Event(enable_timing=True)
        begin.record(stream)
        for _ in range(args.steps):
            for _ in range(total // chunk):
                chunk_call(True)
        finish.record(stream)
        torch.cuda.synchronize()
    ms = begin.elapsed_time(finish) / args.steps
    calls = args.steps * (total // chunk)
    peak, peak_kind = measured_peak()
    h = n // 2 + 1
    # Algorithmic bytes: each image read once and its spectrum written once,
    # with its key, CTF parameters and voltage (the fused kernel's traffic);
    # the separate path also writes and re-reads the standardized image.
    fused_bytes = chunk * (n * n * 4 + n * h * 8 + 8 + 16 + 4)
    std_bytes = chunk * (n * n * 8 + 8)
    fft_bytes = chunk * (n * n * 4 + n * h * 8 + 16 + 4)

    def rate(nbytes, total_ms):
        gbs = nbytes / (total_ms / calls / 1e3) / 1e9
        return {"ms_per_call": total_ms / calls, "achieved_gbs": gbs, "frac": gbs / peak}

    if fused:
        kernels = {"standardize_rfft2": rate(fused_bytes, phase_ms[0])}
        top = kernels["standardize_rfft2"]
    else:
        kernels = {"standardize": rate(std_bytes, phase_ms[0]), "rfft2_ctf": rate(fft_bytes, phase_ms[1])}
        top = kernels["rfft2_ctf"]
    whole_gbs = fused_bytes * (total // chunk) / (ms / 1e3) / 1e9
    line = {
        "metric": f"images/s through standardization + R2C with the CTF epilogue ({n}^2)", "value": total / (ms / 1e3),
        "unit": "images/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"frontend {total} x {n}^2 in chunks of {chunk}, {args.frontend_path}",
                   "l2": f"chunks {chunk * n * n * 4 / 1e9:.2f} GB in, {chunk * n * h * 8 / 1e9:.2f} GB out"},
        "roofline": {"bound": "hbm", "achieved": top["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": top["frac"], "peak_kind": peak_kind,
                     "whole_step": {"bytes_per_image": fused_bytes // chunk, "achieved": whole_gbs,
                                    "frac": whole_gbs / peak}},
        "kernels": kernels,
        "gpu_launches": calls * (1 if fused else 2),
        "clocks": clocks.summary(),
    }
    return line


def run_wiener(args):
    """The Wiener divide + irfft3 of 256^3 accumulators (three passes)."""
    import torch

    from rexlib_b200 import fourier

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    big = 256
    H = big // 2 + 1
    num = torch.randn((big, big, H), dtype=torch.complex64, device=device)
    den = torch.rand((big, big, H), dtype=torch.float32, device=device)
    out = torch.empty((big, big, big), dtype=torch.float32, device=device)
    for _ in range(args.warmup):
        fourier.wiener_irfft3(num, den, 1e-3, out=out)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    begin = torch.cuda.Event(enable_timing=True)
    finish = torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clocks:
        begin.record(stream)
        for _ in range(args.steps):
            fourier.wiener_irfft3(num, den, 1e-3, out=out)
        finish.record(stream)
        torch.cuda.synchronize()
    ms = begin.elapsed_time(finish) / args.steps
    voxels = big * big * H
    # Pass bytes: (12 read + 8 write) + (8 + 8) + (8 read + 4 * N / H write) per complex voxel.
    algorithmic = voxels * (20 + 16 + 8) + big ** 3 * 4
    peak, peak_kind = measured_peak()
    line = {
        "metric": "Wiener divide + irfft3 at 256^3", "value": 1e3 / ms, "unit": "volumes/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "wiener_irfft3 256^3 (constant 1e-3)", "l2": "volumes 101 MB + 67 MB workspace"},
        "roofline": {"bound": "hbm", "achieved": algorithmic / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": algorithmic / (ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind},
        "gpu_launches": args.steps * 3,
        "clocks": clocks.summary(),
    }
    return line


def run_arrays(args):
    """fill, add and divide of complex64 arrays of 2^26 elements (512 MB each,
    well above L2), the elementwise operations callers run between the
    path's steps. The headline is divide; one step is one call."""
    import torch

    from rexlib_b200 import arrays

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    n = 1 << 26
    x = torch.randn(n, dtype=torch.complex64, device=device)
    y = torch.randn(n, dtype=torch.complex64, device=device)
    out = torch.empty_like(x)
    stream = torch.cuda.current_stream()
    calls = {
        "divide": (lambda: arrays.divide(x, y, out=out), 24),
        "add": (lambda: arrays.add(x, y, out=out), 24),
        "fill": (lambda: arrays.fill(out, 1.0), 8),
    }
    rates = {}
    with ClockSampler(0) as clocks:
        for name, (call, bytes_per_element) in calls.items():
            for _ in range(args.warmup):
                call()
            torch.cuda.synchronize()
            begin = torch.cuda.Event(enable_timing=True)
            finish = torch.cuda.Event(enable_timing=True)
            begin.record(stream)
            for _ in range(args.steps):
                call()
            finish.record(stream)
            torch.cuda.synchronize()
            ms = begin.elapsed_time(finish) / args.steps
            rates[name] = (ms, n * bytes_per_element / (ms / 1e3) / 1e9)
    peak, peak_kind = measured_peak()
    ms, gbs = rates["divide"]
    line = {
        "metric": "complex64 divide of 2^26-element arrays", "value": n / (ms / 1e3), "unit": "elements/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
        "config": {"workload": "arrays: divide, add, fill of complex64 x 2^26", "l2": "arrays of 512 MB"},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                     "peak_kind": peak_kind},
        "others": {k: {"ms": v[0], "GB/s": v[1], "frac": v[1] / peak} for k, v in rates.items()},
        "gpu_launches": args.steps * 3,
        "clocks": clocks.summary(),
    }
    return line


def run_pipeline(args):
    """The whole reconstruction step on the GPU: --particles images of --box^2
    (resident, Gaussian noise of mean U[-2,2] and sigma U[0.5,3]) are
    standardized (radius 0.45 n), transformed (R2C) and inserted with their CTF
    (linear window, --mode) into --box^3, in calls of --chunk images;
    then the Wiener divide (1e-3) and C2R of the accumulators. One JSON line
    with the time of each phase."""
    import torch

    from rexlib_b200 import em, fourier

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    n = big = args.box
    P = args.particles
    chunk = min(args.chunk, P)
    h = n // 2 + 1
    H = big // 2 + 1
    g = torch.Generator(device=device)
    g.manual_seed(11)
    images = torch.empty((P, n, n), dtype=torch.float32, device=device)
    images.normal_(generator=g)
    images.mul_(torch.rand((P, 1, 1), generator=g, device=device) * 2.5 + 0.5)
    images.add_(torch.rand((P, 1, 1), generator=g, device=device) * 4 - 2)
    keys = torch.arange(1, P + 1, dtype=torch.int64, device=device)
    tr_h, ctf_h = host_parameters(P, seed=1235)
    transforms = torch.from_numpy(tr_h).to(device)
    ctf = torch.from_numpy(ctf_h).to(device)
    radial = torch.ones(h, dtype=torch.float32, device=device)
    if args.frontend_path is None:
        args.frontend_path = "fused" if n in (64, 128, 256) else "separate"
    fused = args.frontend_path == "fused"
    if fused and n not in (64, 128, 256):
        raise SystemExit("the fused front end runs 64^2, 128^2 and 256^2 images: use --frontend-path separate")
    std = None if fused else torch.empty((chunk, n, n), dtype=torch.float32, device=device)
    spectra = torch.empty((chunk, n, h), dtype=torch.complex64, device=device)
    num = torch.zeros((big, big, H), dtype=torch.complex64, device=device)
    den = torch.zeros((big, big, H), dtype=torch.float32, device=device)
    volume = torch.empty((big, big, big), dtype=torch.float32, device=device)
    window = em.GriddingWindow.linear()
    optics = em.CtfOptics(*OPTICS)
    stream = torch.cuda.current_stream()
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    phase_ms = [0.0, 0.0, 0.0, 0.0]

    def step(timed):
        num.zero_()
        den.zero_()
        for c0 in range(0, P, chunk):
            c1 = min(P, c0 + chunk)
            m = c1 - c0
            if timed:
                marks[0].record(stream)
            if fused:
                # Standardization and R2C in one kernel: marks 1 and 2 coincide.
                fourier.standardize_rfft2_ctf(images[c0:c1], keys[c0:c1], 0.45 * n, (-np.inf, np.inf),
                                              out=spectra[:m])
                if timed:
                    marks[1].record(stream)
            else:
                em.standardize_background_2d(images[c0:c1], keys[c0:c1], 0.45 * n, (-np.inf, np.inf), out=std[:m])
                if timed:
                    marks[1].record(stream)
                fourier.rfft2(std[:m], out=spectra[:m])
            if timed:
                marks[2].record(stream)
            em.insert_ctf_slices(num, den, spectra[:m], transforms[c0:c1], ctf[c0:c1], radial, window, optics,
                                 PIXEL_SIZE, numerator_out=num, denominator_out=den,
                                 deterministic=args.mode == "deterministic")
            if timed:
                marks[3].record(stream)
                marks[3].synchronize()
                phase_ms[0] += marks[0].elapsed_time(marks[1])
                phase_ms[1] += marks[1].elapsed_time(marks[2])
                phase_ms[2] += marks[2].elapsed_time(marks[3])
        if timed:
            marks[3].record(stream)
        fourier.wiener_irfft3(num, den, 1e-3, out=volume)
        if timed:
            marks[4].record(stream)
            marks[4].synchronize()
            phase_ms[3] += marks[3].elapsed_time(marks[4])

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()
    begin = torch.cuda.Event(enable_timing=True)
    finish = torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clocks:
        begin.record(stream)
        for _ in range(args.steps):
            step(False)
        finish.record(stream)
        torch.cuda.synchronize()
    ms = begin.elapsed_time(finish) / args.steps
    step(True)  # one more step, timed phase by phase (synchronizing between phases)
    line = {
        "metric": f"particles/s through standardization, R2C, CTF insertion and the Wiener C2R ({n}^2 into "
                  f"{big}^3)",
        "value": P / (ms / 1e3), "unit": "particles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"pipeline {P} x {n}^2 into {big}^3 in calls of {chunk}, trilinear, {args.mode}, "
                               f"{args.frontend_path} front end",
                   "l2": f"images {P * n * n * 4 / 1e9:.1f} GB > L2, no flush"},
        "phases_ms": ({"standardize_rfft2": phase_ms[0]} if fused else
                      {"standardize": phase_ms[0], "rfft2": phase_ms[1]}) |
                     {"insert_ctf_slices": phase_ms[2], "wiener_irfft3": phase_ms[3]},
        "clocks": clocks.summary(),
    }
    return line


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    others = {"frontend": run_frontend, "wiener": run_wiener, "arrays": run_arrays, "pipeline": run_pipeline,
              "batched": run_batched, "prior": run_prior, "conv3d": run_conv3d, "unet": run_unet}
    if args.workload in others:
        print(json.dumps(others[args.workload](args)), flush=True)
        return

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=device)

    from rexlib_b200 import em

    n = big = args.box
    P = args.particles
    H = big // 2 + 1
    deterministic = args.mode == "deterministic"
    tr_h, ctf_h = host_parameters(P, seed=1234 + rank)
    transforms = torch.from_numpy(tr_h).to(device)
    ctf = torch.from_numpy(ctf_h).to(device)
    radial = torch.ones(n // 2 + 1, dtype=torch.float32, device=device)
    slices = synth_slices(torch, P, n, device, seed=4321 + rank)
    f64 = args.precision == "f64"
    if f64:
        slices = slices.to(torch.complex128)
        transforms, ctf, radial = transforms.double(), ctf.double(), radial.double()
        args.no_e2e = args.no_cpu_baseline = True
    num = torch.zeros((big, big, H), dtype=torch.complex128 if f64 else torch.complex64, device=device)
    den = torch.zeros((big, big, H), dtype=torch.float64 if f64 else torch.float32, device=device)
    window = gpu_window(em, args.window)
    optics = em.CtfOptics(*OPTICS)
    stream = torch.cuda.current_stream()

    def timed_insertion(mode_deterministic: bool, steps: int, warmup: int):
        """Warm-up, then `steps` steps timed on the launching stream: (ms per
        step, whole-job particles/s, mean insertion-call ms, clocks)."""
        for _ in range(warmup):
            num.zero_()
            den.zero_()
            em.insert_ctf_slices(num, den, slices, transforms, ctf, radial, window, optics, PIXEL_SIZE,
                                 numerator_out=num, denominator_out=den, deterministic=mode_deterministic)
        torch.cuda.synchronize()
        kstarts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        begin = torch.cuda.Event(enable_timing=True)
        finish = torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local_rank) as clocks:
            begin.record(stream)
            for i in range(steps):
                num.zero_()
                den.zero_()
                kstarts[i].record(stream)
                em.insert_ctf_slices(num, den, slices, transforms, ctf, radial, window, optics, PIXEL_SIZE,
                                     numerator_out=num, denominator_out=den, deterministic=mode_deterministic)
                ends[i].record(stream)
            finish.record(stream)
            torch.cuda.synchronize()
        if dist:
            dist.barrier()
        launch_ms = [kstarts[i].elapsed_time(ends[i]) for i in range(steps)]
        ms, rate = replica_rate(begin.elapsed_time(finish), steps, P, dist, device)
        return ms, rate, float(np.mean(launch_ms)), clocks.summary()

    # Timed region: K steps, per-launch kernel events on the launching stream.
    ms_per_step, value, avg_launch, clock_summary = timed_insertion(deterministic, args.steps, args.warmup)
    peak, peak_kind = measured_peak()
    real_bytes = 8 if f64 else 4
    algo_bytes = bytes_per_particle(n, big, P, real_bytes) * P
    achieved = algo_bytes / (avg_launch / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "insertion_traffic.json")
    # The committed capture is of the linear window in throughput mode; its
    # traffic per particle scales to this launch when the box matches.
    if os.path.exists(tpath) and args.window == "linear" and not deterministic and not f64:
        with open(tpath) as f:
            t = json.load(f)
        if t.get("box") == big and t.get("dram_bytes_per_particle"):
            traffic = t["dram_bytes_per_particle"] * P
    slices_meta = slices[:1]
    launches = em.insertion_launch_count(num, den, slices_meta, transforms, radial, window, deterministic)
    samples = inserted_samples(n, big) if args.window == "linear" and not f64 else None
    onchip = None
    if samples is not None and clock_summary.get("sm_mhz"):
        onchip = onchip_rates(value / max(1, world), samples, clock_summary["sm_mhz"],
                              stored_taps(tr_h[:32], n, big))
        if not deterministic:
            peaks = onchip_peaks(torch, device)
            onchip.update(peaks)
            onchip["l2_reduction_frac"] = onchip["l2_vector_reductions_per_s"] / peaks["l2_reductions_per_s_measured"]
            onchip["shared_atomic_frac_measured"] = (onchip["shared_atomic_lane_ops_per_s"]
                                                     / peaks["shared_atomic_lane_ops_per_s_measured"])

    # The other configurations, each with its own device timing and clocks
    # (one GPU, rank 0 only): the deterministic mode of this workload, the
    # 10^6 x 128^2 front end, the 64^3 pipeline, the Wiener C2R at 256^3, the
    # 48 batched reconstructions and the learned prior.
    extras = None
    if world == 1 and not args.no_extras and not f64:
        extras = {}
        det_steps = 2
        d_ms, d_value, d_launch, d_clocks = timed_insertion(not deterministic, det_steps, 1)
        other = "throughput" if deterministic else "deterministic"
        extras[other] = {"workload": insertion_config(args, world)["workload"].replace(args.mode, other),
                         "value": d_value, "unit": UNIT, "ms_per_step": d_ms, "steps": det_steps, "warmup": 1,
                         "roofline": {"achieved": algo_bytes / (d_launch / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                      "frac": algo_bytes / (d_launch / 1e3) / 1e9 / peak, "launch_ms": d_launch},
                         "clocks": d_clocks}

    # End to end: host (pinned) inputs copied in chunks, inserted through the
    # public API, accumulators read back, every step.
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(torch, em, args, device, slices, transforms, ctf, radial, window, optics, deterministic,
                      world, dist)
    del slices
    torch.cuda.empty_cache()

    if extras is not None:
        extras.update(run_extra_workloads(args))

    cpu = None
    error_vs_fp64 = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            rate, count, elapsed, kind = reference_sample(P, n, big, 99, 15.0, threads, args.window)
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
                   "sample": f"{count} particles of the workload ({n}^2, CTF, {WINDOWS[args.window][3]}, into {big}^3) in "
                             f"{elapsed:.1f} s on {threads} threads"}
            if n == big == 256 and args.window == "linear":
                error_vs_fp64 = fp64_error_sample(torch, em, device, 2000, threads)
        except Exception as e:  # the checker library is test infrastructure; report its absence
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "port", "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
            "config": insertion_config(args, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "bytes_per_particle": bytes_per_particle(n, big, P, real_bytes), "launch_ms": avg_launch,
                         "onchip": onchip},
            "cpu_baseline": cpu,
            "error_vs_fp64": error_vs_fp64,
            "e2e": e2e,
            "gpu_launches": args.steps * launches,
            "clocks": clock_summary,
            "extra": extras,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def inserted_samples(n: int, big: int) -> int:
    """Samples a particle inserts with unit radial weights and the linear
    window (the +k and -k halves), counted as the kernels and the CPU select
    them: rows |k_y| <= n/2 - 1 (even n), columns 0 .. h - 2, shell
    round(|k|) <= n/2 (row_insertion_kernel.inl:188-226), k_x = 0 once."""
    h = n // 2 + 1
    highest = n // 2 - 1 if n % 2 == 0 else n // 2
    last_column = h - 2 if n % 2 == 0 else h - 1
    ky = np.arange(-highest, highest + 1)[:, None]
    kx = np.arange(0, last_column + 1)[None, :]
    r2 = 4 * (kx * kx + ky * ky)
    last_shell = h - 1
    inside = r2 < (2 * last_shell + 1) ** 2  # round-half-up shell s <= last: 4|k|^2 < (2s + 1)^2
    per_sign = int(inside.sum())
    return 2 * per_sign - int(inside[:, 0].sum())


def stored_taps(transforms: np.ndarray, n: int, big: int) -> tuple[float, float]:
    """(taps, x tap pairs) a particle accumulates into the stored half volume
    with the linear window, averaged over `transforms` (P, 3, 4): every
    inserted sample (inserted_samples' selection, both signs) at K = k_x A0 +
    k_y A1 (rows of the transform, times N/n), its taps floor(K) and
    floor(K) + 1 per axis, kept where x is in [0, N/2] and y, z in
    [-N/2, N/2]. A sample whose K_x is negative reaches the stored half only
    through its other sign, so about half of the inserted samples
    accumulate anything."""
    h = n // 2 + 1
    highest = n // 2 - 1 if n % 2 == 0 else n // 2
    last_column = h - 2 if n % 2 == 0 else h - 1
    ky, kx = np.meshgrid(np.arange(-highest, highest + 1), np.arange(0, last_column + 1), indexing="ij")
    inside = 4 * (kx * kx + ky * ky) < (2 * (h - 1) + 1) ** 2
    kx, ky = kx[inside].astype(np.float64), ky[inside].astype(np.float64)
    half = big // 2
    scale = big / n
    taps = pairs = 0.0
    for t in transforms:
        a, b = t[0, :3].astype(np.float64) * scale, t[1, :3].astype(np.float64) * scale
        for sign in (1.0, -1.0):
            keep = np.ones(kx.shape, bool) if sign > 0 else kx > 0
            K = sign * (kx[keep, None] * a + ky[keep, None] * b)
            f = np.floor(K).astype(np.int64)
            ok = [(f[:, d] + o >= (0 if d == 0 else -half)) & (f[:, d] + o <= half) for d in range(3) for o in (0, 1)]
            in_x = ok[0].astype(np.int64) + ok[1]
            in_y = ok[2].astype(np.int64) + ok[3]
            in_z = ok[4].astype(np.int64) + ok[5]
            taps += float((in_x * in_y * in_z).sum())
            pairs += float(((in_x > 0) * in_y * in_z).sum())
    return taps / len(transforms), pairs / len(transforms)


def onchip_peaks(torch, device) -> dict:
    """The two on-chip rates the tiled insertion's accumulation runs into,
    measured on this device with the library's probe kernels (CUDA events,
    after a warm-up launch): vector FP32 reductions into L2 at random 16-byte
    slots of a 58.5 MB region (the numerator scratch's size), and FP32
    shared-memory atomics at random words of a 48 KB tile (bank conflicts
    included), both at 4 CTAs of 512 threads an SM."""
    import ctypes

    from rexlib_b200 import _capi

    lib = _capi.load()
    stream = torch.cuda.current_stream(device)
    s = ctypes.c_void_p(stream.cuda_stream)
    blocks, threads = 148 * 4, 512
    region_bytes = 58_500_000 // 16 * 16
    region = torch.zeros(region_bytes // 4, dtype=torch.float32, device=device)
    sink = torch.zeros(1, dtype=torch.float32, device=device)

    def timed(run, per_thread, launches=5):
        run(per_thread, 1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for k in range(launches):
            run(per_thread, k + 2)
        b.record(stream)
        torch.cuda.synchronize(device)
        return launches * blocks * threads * per_thread / (a.elapsed_time(b) / 1e3)

    l2 = timed(lambda per, seed: _capi.check(lib.rexlib_b200_l2_reduction_run(
        ctypes.c_void_p(region.data_ptr()), region_bytes, blocks, threads, per, seed, s)), 256)
    shared = timed(lambda per, seed: _capi.check(lib.rexlib_b200_shared_atomic_run(
        ctypes.c_void_p(sink.data_ptr()), blocks, threads, per, seed, s)), 2048)
    del region, sink
    return {"l2_reductions_per_s_measured": l2, "shared_atomic_lane_ops_per_s_measured": shared}


def onchip_rates(particles_per_s: float, samples: int, sm_mhz: float, taps: tuple[float, float] | None = None,
                 sms: int = 148) -> dict:
    """The on-chip work of the linear window's accumulation against its
    nominal rate: each tap that lands in the stored half volume is one
    shared-memory FP32 atomic of the denominator (one lane-op; nominal peak:
    32 lanes an SM a cycle), and each x tap pair one vector L2 reduction of
    the numerator. `taps` is stored_taps' (taps, pairs) per particle; without
    it, every inserted sample counts 8 taps and 4 pairs."""
    per_taps, per_pairs = taps if taps is not None else (8.0 * samples, 4.0 * samples)
    lane_ops = particles_per_s * per_taps
    peak = sms * 32 * sm_mhz * 1e6
    return {"samples_per_particle": samples, "stored_taps_per_particle": per_taps,
            "stored_tap_pairs_per_particle": per_pairs, "shared_atomic_lane_ops_per_s": lane_ops,
            "shared_atomic_peak_nominal": peak, "shared_atomic_frac": lane_ops / peak,
            "l2_vector_reductions_per_s": particles_per_s * per_pairs, "sm_mhz": sm_mhz}


def fp64_error_sample(torch, em, device, count: int, threads: int) -> dict:
    """The error of this workload's GPU result (both modes) and of the CPU
    functor's float32 result against the same insertion in float64 (the
    reference's functor instantiated in double), on `count` particles of
    256^2 into 256^3: relative L2 of numerator and denominator."""
    import oracle

    n = big = 256
    h = H = n // 2 + 1
    tr_h, ctf_h = host_parameters(count, seed=77)
    slices = synth_slices(torch, count, n, device, seed=78)
    host = slices.cpu().numpy()
    tr_d, ctf_d = torch.from_numpy(tr_h).to(device), torch.from_numpy(ctf_h).to(device)
    radial = torch.ones(h, dtype=torch.float32, device=device)
    window, optics = em.GriddingWindow.linear(), em.CtfOptics(*OPTICS)
    gpu = {}
    for mode in ("throughput", "deterministic"):
        num = torch.zeros((big, big, H), dtype=torch.complex64, device=device)
        den = torch.zeros((big, big, H), dtype=torch.float32, device=device)
        em.insert_ctf_slices(num, den, slices, tr_d, ctf_d, radial, window, optics, PIXEL_SIZE, numerator_out=num,
                             denominator_out=den, deterministic=mode == "deterministic")
        gpu[mode] = (num.cpu().numpy(), den.cpu().numpy())
    impl = "ref_fast" if oracle.ref(strict=False) is not None else "oracle"
    kw = dict(window=oracle.Window("linear"), optics=oracle.Optics(*OPTICS), pixel_size=PIXEL_SIZE,
              implementation=impl, threads=threads)
    num64 = np.zeros((1, big, big, H), np.complex128)
    den64 = np.zeros((1, big, big, H), np.float64)
    oracle.insert("ctf", num64, den64, host.astype(np.complex128), tr_h[None].astype(np.float64),
                  np.ones(h, np.float64), ctf_h[None].astype(np.float64), **kw)
    num32 = np.zeros((1, big, big, H), np.complex64)
    den32 = np.zeros((1, big, big, H), np.float32)
    oracle.insert("ctf", num32, den32, host, tr_h[None], np.ones(h, np.float32), ctf_h[None], **kw)

    def rel(a, b):
        a = np.asarray(a, np.complex128 if np.iscomplexobj(a) else np.float64)
        return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))

    out = {"sample": f"{count} particles of 256^2 into 256^3, CTF, trilinear; float64: the reference functor in "
                     f"double ({impl})",
           "cpu_float32": {"numerator": rel(num32[0], num64[0]), "denominator": rel(den32[0], den64[0])}}
    for mode, (num, den) in gpu.items():
        out[f"gpu_{mode}"] = {"numerator": rel(num, num64[0]), "denominator": rel(den, den64[0]),
                              "vs_cpu_float32_numerator": rel(num, num32[0]),
                              "vs_cpu_float32_denominator": rel(den, den32[0])}
    return out


def batched_job_set(seed: int = 2024, jobs: int = 48):
    """The ragged job set of the batched reconstructions: per job a box
    n = N drawn from {96, 128, 160, 200, 256} and a particle count drawn
    lognormal around a median of 8,000, clipped to [2,000, 40,000]."""
    rng = np.random.default_rng(seed)
    boxes = rng.choice([96, 128, 160, 200, 256], size=jobs)
    counts = np.clip(np.round(np.exp(rng.normal(np.log(8000.0), 0.8, size=jobs))), 2000, 40000).astype(int)
    return [(int(b), int(c)) for b, c in zip(boxes, counts)]


def run_batched(args):
    """48 ragged reconstructions (CTF, trilinear, throughput mode): one
    batched call (after its tuner has settled, replayed from a CUDA graph)
    against one insert_ctf_slices call per job, on the same resident inputs;
    the accumulators of both compared."""
    import torch

    from rexlib_b200 import em

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    spec = batched_job_set()
    jobs = []
    g = torch.Generator(device=device)
    g.manual_seed(31)
    for i, (n, p) in enumerate(spec):
        h = n // 2 + 1
        tr, ctf = host_parameters(p, seed=500 + i)
        slices = torch.complex(torch.randn((p, n, h), generator=g, device=device),
                               torch.randn((p, n, h), generator=g, device=device))
        jobs.append(dict(numerator=torch.zeros((1, n, n, h), dtype=torch.complex64, device=device),
                         denominator=torch.zeros((1, n, n, h), dtype=torch.float32, device=device),
                         slices=slices, transforms=torch.from_numpy(tr).to(device)[None],
                         ctf=torch.from_numpy(ctf).to(device)[None],
                         radial_weights=torch.ones(h, dtype=torch.float32, device=device)))
    window, optics = em.GriddingWindow.linear(), em.CtfOptics(*OPTICS)
    particles = sum(p for _, p in spec)
    batch = em.BatchedInsertion(jobs, window, "ctf", optics, PIXEL_SIZE, deterministic=False)
    stream = torch.cuda.Stream(device)

    def zero():
        for j in jobs:
            j["numerator"].zero_()
            j["denominator"].zero_()

    with torch.cuda.stream(stream):
        for _ in range(12):  # the tuner tries its candidates, then settles
            zero()
            batch()
        torch.cuda.synchronize()
        tuned, config = batch.tuning()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            batch()

        def sequential():
            for j in jobs:
                em.insert_ctf_slices(j["numerator"], j["denominator"], j["slices"], j["transforms"], j["ctf"],
                                     j["radial_weights"], window, optics, PIXEL_SIZE, numerator_out=j["numerator"],
                                     denominator_out=j["denominator"], deterministic=False)

        def timed(call, steps):
            for _ in range(args.warmup):
                zero()
                call()
            torch.cuda.synchronize()
            total = 0.0
            with ClockSampler(0) as clocks:
                for _ in range(steps):
                    zero()
                    a = torch.cuda.Event(enable_timing=True)
                    b = torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    call()
                    b.record(stream)
                    b.synchronize()
                    total += a.elapsed_time(b)
            return total / steps, clocks.summary()

        seq_ms, seq_clocks = timed(sequential, args.steps)
        seq_out = [(j["numerator"].clone(), j["denominator"].clone()) for j in jobs]
        bat_ms, bat_clocks = timed(graph.replay, args.steps)
    torch.cuda.synchronize()

    def rel(a, b):
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

    worst = max(max(rel(j["numerator"], n), rel(j["denominator"], d)) for j, (n, d) in zip(jobs, seq_out))
    del graph
    peak, peak_kind = measured_peak()
    algo = sum(bytes_per_particle(n, n, p) * p for n, p in spec)
    return {
        "metric": "particles/s, 48 ragged reconstructions in one batched call (CUDA graph) vs one call per job",
        "value": particles / (bat_ms / 1e3), "unit": "particles/s", "ms_per_step": bat_ms, "steps": args.steps,
        "warmup": args.warmup,
        "config": {"workload": f"batched insert_ctf_slices, 48 jobs, boxes {{96..256}}, {particles} particles, "
                               "trilinear, throughput"},
        "sequential": {"value": particles / (seq_ms / 1e3), "ms_per_step": seq_ms, "clocks": seq_clocks},
        "speedup_vs_sequential": seq_ms / bat_ms,
        "max_rel_l2_vs_sequential": worst,
        "tuner": {"tuned": tuned, "tile_cells": config[0], "min_hits": config[1], "max_hits": config[2]},
        "roofline": {"bound": "hbm", "achieved": algo / (bat_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": algo / (bat_ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind},
        "gpu_launches": args.steps * batch.launch_count(),
        "clocks": bat_clocks,
    }


PRIOR_SIGMA = (2.0, 8.0)  # blob widths in voxels, training and evaluation phantoms
PRIOR_WEIGHT = 6.0  # prior weight (times the mean denominator) of the iterates shown in training


def run_prior(args):
    """The learned prior (3D U-Net, 16-32-64-128), trained and applied on the
    library's kernels:
    - training pairs generated on the GPU: Wiener maps of seeded blob and
      helical-filament phantoms (20-200 blobs, sigma 2-8 voxels) of extent
      `--prior-extent` from 2,000-20,000 noisy particles at SNR 0.05-0.2,
      against the phantom low-passed to half Nyquist;
    - Adam training on the library's forward and backward kernels: first on
      the Wiener maps, then with every other input one of the network's own
      regularised iterates (1 to --iterate-depth iterations), so that it
      stays accurate along the iteration it serves in;
    - evaluation on an unseen phantom at `--eval-extent` (200 blobs, sigma
      2-8 voxels, SNR 0.1): the FSC-0.143 shell against the phantom of the
      plain Wiener map at 100% and 50% of the particles and of the
      learned-prior reconstruction (10 iterations; the best of four prior
      weights at 50%, applied at 100%) and of one iteration at that weight;
      the gate keeps the plain map where the prior does not raise the shell;
    - the tensor-core convolution's throughput against the measured BF16
      peak, and the forward pass at both extents."""
    import torch

    from rexlib_b200 import prior

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    e, E = args.prior_extent, args.eval_extent
    stream = torch.cuda.current_stream()

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    t0 = time.perf_counter()
    inputs, targets, nums, dens = prior.make_pairs(args.pairs, e, seed=2024, blobs=(20, 200), sigma=PRIOR_SIGMA,
                                                   accumulators=True)
    torch.cuda.synchronize()
    pair_s = time.perf_counter() - t0
    net = prior.UNet(e, seed=1)
    a, b = events()
    a.record(stream)
    losses = prior.train(net, inputs, targets, args.train_steps, 1e-3)
    b.record(stream)
    torch.cuda.synchronize()
    train_ms = a.elapsed_time(b)
    a.record(stream)
    losses += prior.train_on_iterates(net, inputs, targets, nums, dens, args.iterate_steps, PRIOR_WEIGHT,
                                      max_iterations=args.iterate_depth, average_from=args.average_from)
    b.record(stream)
    torch.cuda.synchronize()
    iterate_ms = a.elapsed_time(b)
    del inputs, targets, nums, dens
    torch.cuda.empty_cache()

    # Evaluation on a phantom the network has not seen, at the evaluation
    # extent (the network is convolutional: its weights apply at any extent).
    evaluator = net if E == e else prior.UNet(E, seed=1)
    if evaluator is not net:
        evaluator.load(net.parameters())
    rng = np.random.default_rng(99)
    blobs = prior.blob_phantom(rng, E, args.eval_blobs, sigma=PRIOR_SIGMA)
    full = prior.Dataset(blobs, E, args.eval_particles, 0.1, seed=100)
    half = prior.Dataset(blobs, E, args.eval_particles // 2, 0.1, seed=100)
    plain_full, _ = full.resolution(full.wiener())
    plain_half, _ = half.resolution(half.wiener())
    learned = {}
    base = float(half.den.mean())
    a, b = events()
    a.record(stream)
    for factor in (6.0, 8.0, 12.0, 16.0):
        learned[factor], _ = half.resolution(prior.regularised(evaluator, half, 10, factor * base))
    b.record(stream)
    torch.cuda.synchronize()
    regularised_ms = a.elapsed_time(b) / 4
    best = max(learned, key=learned.get)
    learned_full, _ = full.resolution(prior.regularised(evaluator, full, 10, best * float(full.den.mean())))
    once_half, _ = half.resolution(prior.regularised(evaluator, half, 1, best * base))
    once_full, _ = full.resolution(prior.regularised(evaluator, full, 1, best * float(full.den.mean())))
    del full, half
    torch.cuda.empty_cache()

    # Throughput: one 64 -> 64 tensor-core convolution at 128^3, and the
    # network's forward pass at both extents.
    peak = 1666.7
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
    except (OSError, KeyError, ValueError):
        pass
    x = torch.randn((128, 128, 128, 64), device=device).to(torch.bfloat16)
    w = (torch.randn((64, 27, 64), device=device) * 0.05).to(torch.bfloat16)
    y = torch.empty_like(x)
    for _ in range(3):
        prior.conv3d([x], w, None, prior.EPILOGUE_NONE, out=[y])
    a, b = events()
    a.record(stream)
    for _ in range(20):
        prior.conv3d([x], w, None, prior.EPILOGUE_NONE, out=[y])
    b.record(stream)
    torch.cuda.synchronize()
    conv_ms = a.elapsed_time(b) / 20
    conv_tflops = 2.0 * 27 * 64 * 64 * 128 ** 3 / (conv_ms / 1e3) / 1e12
    del x, y
    forward = {}
    for extent, n2 in ((e, net), (E, evaluator)):
        v = torch.randn((extent,) * 3, device=device)
        out = torch.empty_like(v)
        for _ in range(2):
            n2.forward(v, out)
        a, b = events()
        a.record(stream)
        for _ in range(5):
            n2.forward(v, out)
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / 5
        forward[str(extent)] = {"ms": ms, "tflops": prior.conv_flops(extent) / (ms / 1e3) / 1e12}
    if evaluator is not net:
        evaluator.close()
    net.close()
    reaches = learned[best] >= plain_full
    return {
        "metric": "FSC-0.143 shell against the phantom: learned prior at 50% of the particles vs plain Wiener",
        "value": learned[best], "unit": "shell", "higher_is_better": True,
        "config": {"workload": f"U-Net prior trained at {e}^3 ({args.pairs} pairs, {args.train_steps} Adam steps "
                               f"+ {args.iterate_steps} with its own iterates), "
                               f"regularised reconstruction at {E}^3 from {args.eval_particles} particles at SNR 0.1 "
                               f"(50%: {args.eval_particles // 2})"},
        "plain_wiener": {"100%": plain_full, "50%": plain_half},
        "learned_prior": {"50%": learned[best], "100%": learned_full, "weight_factor": best,
                          "weights_tried": {str(k): v for k, v in learned.items()},
                          "ms_per_reconstruction": regularised_ms,
                          "one_iteration": {"50%": once_half, "100%": once_full}},
        "learned_at_50_reaches_plain_at_100": reaches,
        "gate": {"50%": "learned" if learned[best] > plain_half else "plain",
                 "100%": "learned" if learned_full > plain_full else "plain"},
        "training": {"pairs_s": pair_s, "ms_per_step": train_ms / max(1, args.train_steps),
                     "ms_per_iterate_step": iterate_ms / max(1, args.iterate_steps), "losses": losses[::4]},
        "tensor_core": {"conv3d_64to64_128cubed_ms": conv_ms, "tflops": conv_tflops, "peak": peak,
                        "frac": conv_tflops / peak},
        "forward": forward,
    }


def bf16_peak() -> float:
    """The measured dense BF16 peak (TFLOP/s, burst), else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"])
    except (OSError, KeyError, ValueError):
        return 1590.0


def run_conv3d(args):
    """One 3x3x3 tensor-core convolution of random BF16 volumes at
    --prior-extent with --conv-channels, timed over --steps launches after
    --warmup (the inputs, larger than L2 from 64 channels at 128^3, stay
    resident)."""
    import torch

    from rexlib_b200 import prior

    torch.cuda.set_device(0)
    cin, cout = (int(c) for c in args.conv_channels.split(","))
    e = args.prior_extent
    x = torch.randn((e, e, e, cin), device="cuda").to(torch.bfloat16)
    w = (torch.randn((cout, 27, cin), device="cuda") / (27 * cin) ** 0.5).to(torch.bfloat16)
    y = torch.empty((e, e, e, cout), dtype=torch.bfloat16, device="cuda")
    error = torch.zeros(1, dtype=torch.int32, device="cuda")
    if args.conv_pass == "wgrad":
        # The weight and bias gradients for an output gradient y.
        y.copy_(torch.randn((e, e, e, cout), device="cuda"))
        dw = torch.zeros((cout, 27, cin), dtype=torch.float32, device="cuda")
        db = torch.zeros(cout, dtype=torch.float32, device="cuda")

        def launch():
            prior.conv3d_wgrad([x], y, dw, db, error=error)
    else:
        def launch():
            prior.conv3d([x], w, None, prior.EPILOGUE_NONE, out=[y], error=error)
    for _ in range(args.warmup):
        launch()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        launch()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    tflops = 2.0 * 27 * cin * cout * e ** 3 / (ms / 1e3) / 1e12
    peak = bf16_peak()
    what = "3x3x3 convolution" if args.conv_pass == "forward" else "3x3x3 convolution weight gradient"
    return {"metric": what + " TFLOP/s (BF16 operands, FP32 accumulation)", "value": tflops,
            "unit": "TFLOP/s", "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": f"conv3d{'' if args.conv_pass == 'forward' else ' wgrad'} {cin}->{cout} channels "
                                   f"at {e}^3"},
            "roofline": {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s", "frac": tflops / peak},
            "wait_errors": int(error.item())}


def run_unet(args):
    """The U-Net prior's forward pass (or, with --train, a training step:
    forward, backward and Adam) at --prior-extent on a random volume, timed
    over --steps after --warmup."""
    import torch

    from rexlib_b200 import prior

    torch.cuda.set_device(0)
    e = args.prior_extent
    net = prior.UNet(e, seed=1)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((e,) * 3, device="cuda", generator=g)
    t = torch.randn((e,) * 3, device="cuda", generator=g)
    out = torch.empty_like(x)

    def step():
        net.forward(x, out)
        if args.train:
            net.backward(t)
            net.step(1e-4)

    for _ in range(args.warmup):
        step()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        step()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    error = net.error()
    net.close()
    flops = prior.conv_flops(e) * (3 if args.train else 1)
    return {"metric": "U-Net " + ("training step" if args.train else "forward pass") + " time", "value": ms,
            "unit": "ms", "higher_is_better": False, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": f"U-Net 16-32-64-128 at {e}^3, " + ("training step" if args.train else "forward")},
            "convolution_tflops": flops / (ms / 1e3) / 1e12, "wait_errors": error}


def run_extra_workloads(args) -> dict:
    """The front end (10^6 x 128^2), the 64^3 pipeline of 1,000 particles and
    the Wiener C2R at 256^3, each timed as its own workload; the compact part
    of each line."""
    import copy

    def compact(line):
        keep = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "roofline", "clocks", "phases_ms",
                "kernels", "gpu_launches")
        out = {k: line[k] for k in keep if k in line}
        out["workload"] = line["config"]["workload"]
        return out

    extras = {}
    a = copy.copy(args)
    a.images, a.chunk, a.image_box, a.frontend_path, a.steps, a.warmup = 1_000_000, 100_000, 128, None, 3, 2
    extras["frontend"] = compact(run_frontend(a))
    a = copy.copy(args)
    a.box, a.particles, a.chunk, a.mode, a.frontend_path, a.steps, a.warmup = 64, 1000, 1000, "throughput", None, 600, 5
    extras["pipeline_cfg0"] = compact(run_pipeline(a))
    a = copy.copy(args)
    a.steps, a.warmup = 4000, 5
    extras["wiener_256"] = compact(run_wiener(a))
    a = copy.copy(args)
    a.steps, a.warmup = 3, 1
    line = run_batched(a)
    extras["batched_cfg3"] = compact(line) | {k: line[k] for k in ("sequential", "speedup_vs_sequential",
                                                                   "max_rel_l2_vs_sequential", "tuner")}
    a = copy.copy(args)
    line = run_prior(a)
    extras["prior_cfg4"] = {k: line[k] for k in ("metric", "value", "unit", "config", "plain_wiener", "learned_prior",
                                                 "learned_at_50_reaches_plain_at_100", "gate", "training",
                                                 "tensor_core", "forward")}
    return extras


def replica_rate(total_ms: float, steps: int, particles: int, dist=None, device=None) -> tuple[float, float]:
    """(ms per step, whole-job particles/s) of the replicas: every rank
    inserted `particles` per step, and the job takes as long as its slowest
    rank (the maximum over ranks of each rank's device-timed region)."""
    import torch

    world = 1
    if dist is not None and dist.is_initialized():
        world = dist.get_world_size()
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / steps
    return ms_per_step, world * particles / (ms_per_step / 1e3)


def run_e2e(torch, em, args, device, slices, transforms, ctf, radial, window, optics, deterministic, world, dist):
    P = args.particles
    chunk = 8192
    host = torch.empty(slices.shape, dtype=slices.dtype, pin_memory=True)
    host.copy_(slices)
    del slices
    torch.cuda.empty_cache()
    tr_host = transforms.cpu().pin_memory()
    ctf_host = ctf.cpu().pin_memory()
    big = args.box
    H = big // 2 + 1
    num = torch.zeros((big, big, H), dtype=torch.complex64, device=device)
    den = torch.zeros((big, big, H), dtype=torch.float32, device=device)
    num_host = torch.empty(num.shape, dtype=num.dtype, pin_memory=True)
    den_host = torch.empty(den.shape, dtype=den.dtype, pin_memory=True)
    buffers = [torch.empty((chunk,) + tuple(host.shape[1:]), dtype=host.dtype, device=device) for _ in range(2)]
    copy_stream = torch.cuda.Stream(device)
    compute = torch.cuda.current_stream()
    copied = [torch.cuda.Event() for _ in range(2)]
    consumed = [torch.cuda.Event() for _ in range(2)]

    def e2e_step():
        num.zero_()
        den.zero_()
        tr_dev = tr_host.to(device, non_blocking=True)
        ctf_dev = ctf_host.to(device, non_blocking=True)
        for i, start in enumerate(range(0, P, chunk)):
            stop = min(P, start + chunk)
            b = i % 2
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(consumed[b])
                buffers[b][: stop - start].copy_(host[start:stop], non_blocking=True)
                copied[b].record(copy_stream)
            compute.wait_event(copied[b])
            em.insert_ctf_slices(num, den, buffers[b][: stop - start], tr_dev[start:stop], ctf_dev[start:stop],
                                 radial, window, optics, PIXEL_SIZE, numerator_out=num, denominator_out=den,
                                 deterministic=deterministic)
            consumed[b].record(compute)
        num_host.copy_(num, non_blocking=True)
        den_host.copy_(den, non_blocking=True)

    for b in range(2):
        consumed[b].record(compute)
    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    begin = torch.cuda.Event(enable_timing=True)
    finish = torch.cuda.Event(enable_timing=True)
    begin.record(compute)
    for _ in range(args.steps):
        e2e_step()
    finish.record(compute)
    torch.cuda.synchronize()
    _, rate = replica_rate(begin.elapsed_time(finish), args.steps, P, dist, device)
    h2d = host.numel() * 8 + tr_host.numel() * 4 + ctf_host.numel() * 4
    d2h = num.numel() * 8 + den.numel() * 4
    return {"value": rate, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}


if __name__ == "__main__":
    main()
