"""Batched reconstructions on the B200: many insertions of uneven box size
and particle count in one set of launches (rexlib_b200_batched_insert), one
persistent launch claiming every job's work items.

- Deterministic mode: each job's accumulators are the bits of one
  insert_*_slices call on its operands, and (plain and weighted kinds) the
  bits of the reference CPU functor.
- Throughput mode: each job within relative L2 1e-5 of the oracle.
- Captured in a CUDA graph and replayed: the bits of the eager call
  (deterministic mode).
- The online tuner: the first calls of a job set try the candidate tile
  settings, later calls take the fastest, and REXLIB_B200_TUNE_CACHE keeps
  the choice for another process."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import _capi, em
from tests.cases import insertion_inputs, rel_l2
from tests.test_insertion_gpu import PIXEL, WINDOWS, gpu_insert

pytestmark = pytest.mark.gpu

OPTICS = em.CtfOptics(300.0, 2.7, 0.1)
ORACLE_OPTICS = oracle.Optics(300.0, 2.7, 0.1)
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (n, N, particles, volumes): boxes and counts that differ from job to job,
# odd and even, N != n, one job of two volumes.
SHAPES = [(32, 32, 60, 1), (24, 40, 35, 1), (33, 33, 80, 1), (48, 48, 20, 2), (40, 24, 50, 1), (64, 64, 90, 1),
          (17, 17, 30, 1)]


def cases(kind, seed):
    return [insertion_inputs(n, big, p, volumes=v, kind=kind, seed=seed + 13 * i, radial_per_particle=True)
            for i, (n, big, p, v) in enumerate(SHAPES)]


def gpu_job(c, kind):
    to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    V = c["numerator"].shape[0]
    job = dict(numerator=to(c["numerator"].reshape(V, 1, *c["numerator"].shape[1:])),
               denominator=to(c["denominator"].reshape(V, 1, *c["denominator"].shape[1:])),
               slices=to(c["slices"]), transforms=to(c["transforms"]), radial_weights=to(c["radial"]))
    if kind == "ctf":
        job["ctf"] = to(c["extra"])
    elif kind == "weighted":
        job["weights"] = to(c["extra"])
    return job


def host(job, c):
    shape = c["numerator"].shape
    return job["numerator"].cpu().numpy().reshape(shape), job["denominator"].cpu().numpy().reshape(shape)


def oracle_insert(kind, c, window_name):
    num, den = c["numerator"].copy(), c["denominator"].copy()
    oracle.insert(kind, num, den, c["slices"], c["transforms"], c["radial"], c["extra"], window=WINDOWS[window_name][1],
                  optics=ORACLE_OPTICS, pixel_size=PIXEL)
    return num, den


@pytest.mark.parametrize("kind", ["plain", "ctf", "weighted"])
@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb2"])
def test_deterministic_batch_equals_one_call_per_job(kind, window_name):
    cs = cases(kind, 700)
    jobs = [gpu_job(c, kind) for c in cs]
    batch = em.BatchedInsertion(jobs, WINDOWS[window_name][0], kind, OPTICS, PIXEL, deterministic=True)
    batch()
    torch.cuda.synchronize()
    for c, job in zip(cs, jobs):
        num, den = host(job, c)
        want_num, want_den, _, _ = gpu_insert(kind, c, WINDOWS[window_name][0], deterministic=True)
        np.testing.assert_array_equal(num, want_num)
        np.testing.assert_array_equal(den, want_den)
        if kind != "ctf":
            onum, oden = oracle_insert(kind, c, window_name)
            np.testing.assert_array_equal(num, onum)
            np.testing.assert_array_equal(den, oden)


@pytest.mark.parametrize("kind", ["plain", "ctf", "weighted"])
@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb15", "kb2"])
def test_throughput_batch_matches_the_oracle(kind, window_name):
    cs = cases(kind, 800)
    jobs = [gpu_job(c, kind) for c in cs]
    batch = em.BatchedInsertion(jobs, WINDOWS[window_name][0], kind, OPTICS, PIXEL, deterministic=False)
    batch()
    torch.cuda.synchronize()
    for c, job in zip(cs, jobs):
        num, den = host(job, c)
        onum, oden = oracle_insert(kind, c, window_name)
        assert rel_l2(num, onum) <= 1e-5 and rel_l2(den, oden) <= 1e-5, (kind, window_name, c["numerator"].shape)


def test_every_tuner_candidate_gives_the_same_insertion(monkeypatch, tmp_path):
    # The calls that try the candidates each insert exactly: every job
    # within 1e-5 of the oracle after every call.
    monkeypatch.setenv("REXLIB_B200_TUNE_CACHE", str(tmp_path / "unused"))
    cs = cases("ctf", 900)
    for call in range(8):
        jobs = [gpu_job(c, "ctf") for c in cs]
        batch = em.BatchedInsertion(jobs, WINDOWS["linear"][0], "ctf", OPTICS, PIXEL, deterministic=False)
        batch()
        torch.cuda.synchronize()
        for c, job in zip(cs, jobs):
            num, den = host(job, c)
            onum, oden = oracle_insert("ctf", c, "linear")
            assert rel_l2(num, onum) <= 1e-5 and rel_l2(den, oden) <= 1e-5, call


def test_batch_replays_from_a_cuda_graph():
    cs = cases("ctf", 1000)
    jobs = [gpu_job(c, "ctf") for c in cs]
    start = [(j["numerator"].clone(), j["denominator"].clone()) for j in jobs]
    batch = em.BatchedInsertion(jobs, WINDOWS["linear"][0], "ctf", OPTICS, PIXEL, deterministic=True)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        batch()  # eager, on the capture stream
    torch.cuda.synchronize()
    eager = [(j["numerator"].clone(), j["denominator"].clone()) for j in jobs]
    for j, (n0, d0) in zip(jobs, start):
        j["numerator"].copy_(n0)
        j["denominator"].copy_(d0)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        batch()
    for replay in range(2):
        for j, (n0, d0) in zip(jobs, start):
            j["numerator"].copy_(n0)
            j["denominator"].copy_(d0)
        graph.replay()
        torch.cuda.synchronize()
        for j, (n1, d1) in zip(jobs, eager):
            assert torch.equal(j["numerator"], n1) and torch.equal(j["denominator"], d1), replay


def test_tuner_settles_and_its_choice_persists(tmp_path):
    # A job set of its own (so no earlier test has tuned it): the calls try
    # the candidates, the tuner settles on one, writes it to the cache file,
    # and a new process reads it back as already tuned.
    cache = tmp_path / "tune.txt"
    script = f"""
import os, sys, json
os.environ["REXLIB_B200_TUNE_CACHE"] = {str(cache)!r}
sys.path.insert(0, {ROOT!r})
import torch
from rexlib_b200 import em
from tests.test_batched_gpu import gpu_job, OPTICS, PIXEL
from tests.test_insertion_gpu import WINDOWS
from tests.cases import insertion_inputs
cs = [insertion_inputs(n, n, p, kind="ctf", seed=i) for i, (n, p) in enumerate([(56, 70), (72, 40), (40, 90)])]
jobs = [gpu_job(c, "ctf") for c in cs]
batch = em.BatchedInsertion(jobs, WINDOWS["linear"][0], "ctf", OPTICS, PIXEL, deterministic=False)
states = [batch.tuning()[0]]
for _ in range(int(sys.argv[1])):
    batch()
    torch.cuda.synchronize()
states.append(batch.tuning()[0])
print(json.dumps({{"states": states, "config": batch.tuning()[1]}}))
"""
    first = subprocess.run([sys.executable, "-c", script, "8"], capture_output=True, text=True, timeout=600)
    assert first.returncode == 0, first.stderr
    got = json.loads(first.stdout.strip().splitlines()[-1])
    assert got["states"] == [False, True]
    assert cache.exists() and len(cache.read_text().splitlines()) == 1
    second = subprocess.run([sys.executable, "-c", script, "0"], capture_output=True, text=True, timeout=600)
    assert second.returncode == 0, second.stderr
    again = json.loads(second.stdout.strip().splitlines()[-1])
    assert again["states"] == [True, True] and again["config"] == got["config"]


def test_batched_call_refuses_what_it_does_not_run():
    c = insertion_inputs(16, 16, 4, kind="ctf", seed=1)
    jobs = [gpu_job(c, "ctf")]
    # Kaiser-Bessel half-widths above 2: the batched kernels' table is for
    # half-widths up to 2.
    with pytest.raises(_capi.RexlibB200Error, match="half-widths up to 2"):
        em.BatchedInsertion(jobs, em.GriddingWindow.kaiser_bessel(3.0, 10.0), "ctf", OPTICS, PIXEL)
    with pytest.raises(_capi.RexlibB200Error, match="1 to 64 jobs"):
        em.BatchedInsertion([gpu_job(c, "ctf") for _ in range(65)], WINDOWS["linear"][0], "ctf", OPTICS, PIXEL)
